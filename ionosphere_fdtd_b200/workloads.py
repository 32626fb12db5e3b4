"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No dataset is involved: each configuration is a parameterised Earth-ionosphere
setup (material profile, plasma profile, source, receivers) built from a seed.

* ``config1``: s2 / 24 cells, ground sigma 1e-2 S/m, air sigma 0 below 50 km
  and 1e-7 exp((h - 60 km)/4 km) S/m capped at 1e-3 above, one vertical 20 Hz
  Gaussian current at a seed-chosen vertex, 8 seed-uniform surface receivers
  (mesh level and radial cells can be raised: the fused-step comparison runs
  it at s9 / 80).
* ``config2``: s7 / 40 cells, FP32, the config-1 conductivity plus a Drude
  electron plasma n_e(h) = 1e6 exp((h - 85 km)/3 km) m^-3,
  nu(h) = 1e7 exp(-(h - 70 km)/6 km) s^-1, a 50 Hz source and 64 receivers at
  seed-uniform sphere points with barycentric weights.
* ``config3``: an ensemble of 64 independent runs of uneven size: subdivision
  uniform in {5, 6, 7}, radial cells uniform in 24-60, an exponential
  ionosphere sigma(h) = sigma0 exp((h - h0)/zeta) with sigma0 log-uniform in
  1e-8-1e-6 S/m, h0 uniform in 55-70 km and zeta uniform in 3-6 km, ground
  sigma log-uniform in 1e-3-1e-1 S/m, a seed-uniform source vertex with a
  carrier uniform in 10-60 Hz and 16 receivers at seed-uniform sphere points.
* ``config4``: s9 / 80 cells over 0-100 km with the surface-impedance lower
  boundary over a seeded smooth log-normal ground-conductivity map (median
  1e-2 S/m), the config-2 plasma, a 20 Hz source and 256 receivers.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .plasma import ELECTRON_MASS_KG, ELEMENTARY_CHARGE_C, ColdPlasmaSpecies, MeshPlasmaModel
from .provenance import DatasetProvenance, VariableProvenance
from .sources import GaussianCurrent, geographic_distribution


class ProfileMaterial:
    """Volume ground below 0 m; exponential air conductivity above a cutoff."""

    def __init__(self, ground_sigma=1.0e-2, ground_eps=10.0, cutoff_m=50_000.0, prefactor=1.0e-7, h0_m=60_000.0, zeta_m=4_000.0, cap=1.0e-3):
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


def synthetic_provenance() -> DatasetProvenance:
    return DatasetProvenance(
        dataset_id="synthetic.profile-plasma.v1",
        title="Seeded synthetic Drude plasma profile",
        version="1",
        source_url="https://example.invalid/synthetic-plasma",
        citation="Synthetic benchmark input.",
        license="CC0-1.0",
        retrieved_at="2026-12-01T00:00:00Z",
        source_sha256="0" * 64,
        coordinate_reference_system="geocentric Cartesian",
        variables=(
            VariableProvenance("B", "T", "T", "identity"),
            VariableProvenance("number_density", "m^-3", "m^-3", "identity"),
            VariableProvenance("collision_frequency", "Hz", "Hz", "identity"),
        ),
    )


def drude_profile_plasma(mesh, midpoint_altitudes_m) -> MeshPlasmaModel:
    """Altitude-only electron plasma, B = 0 (broadcast arrays, no per-face copies)."""

    h = np.asarray(midpoint_altitudes_m, dtype=np.float64)
    shape = (mesh.n_faces, len(h))
    density = np.broadcast_to(1.0e6 * np.exp((h - 85_000.0) / 3_000.0), shape)
    collision = np.broadcast_to(1.0e7 * np.exp(-(h - 70_000.0) / 6_000.0), shape)
    magnetic = np.broadcast_to(np.zeros((1, len(h), 3)), (*shape, 3))
    electron = ColdPlasmaSpecies("electron", -ELEMENTARY_CHARGE_C, ELECTRON_MASS_KG, density, collision)
    return MeshPlasmaModel.from_mesh(mesh, h, magnetic, (electron,), provenance=(synthetic_provenance(),), interpolation="altitude profile")


def smooth_log_normal(directions, seed: int, median: float = 1.0e-2, spread: float = 0.5):
    """Seeded smooth field (Gaussian-weighted monomials of degree <= 3) made log-normal."""

    d = np.asarray(directions, dtype=np.float64)
    rng = np.random.default_rng(seed)
    x, y, z = (np.ascontiguousarray(d[:, k]) for k in range(3))
    terms = (
        lambda: x, lambda: y, lambda: z, lambda: x * y, lambda: y * z, lambda: z * x, lambda: x * x - y * y,
        lambda: 3 * z * z - 1, lambda: x * y * z, lambda: x**3 - 3 * x * y * y, lambda: z**3,
    )
    weights = rng.standard_normal(len(terms))
    # the weighted sum of the monomials, one term at a time (no (n, 11) basis matrix)
    field = np.zeros(len(d))
    for w, term in zip(weights, terms):
        field += w * term()
    field = (field - field.mean()) / max(field.std(), 1e-30)
    return median * np.exp(spread * field)


def vertex_lat_lon(vertices, index: int) -> tuple[float, float]:
    v = np.asarray(vertices)[index]
    return float(np.degrees(np.arcsin(np.clip(v[2], -1.0, 1.0)))), float(np.degrees(np.arctan2(v[1], v[0])))


def uniform_receivers(simulation, count: int, seed: int, altitude_m: float = 0.0):
    """``count`` seed-uniform sphere points as barycentric Er receivers."""

    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, count)
    lon = rng.uniform(-180.0, 180.0, count)
    lat = np.degrees(np.arcsin(z))
    rows = [geographic_distribution(simulation, float(a), float(o), altitude_m) for a, o in zip(lat, lon)]
    vertices = np.stack([r[0] for r in rows]).astype(np.int64)
    layers = np.asarray([r[1] for r in rows], dtype=np.int64)
    weights = np.stack([r[2] for r in rows])
    return vertices, layers, weights


@dataclass
class Workload:
    name: str
    simulation: object
    receivers: tuple
    cells: int
    bytes_per_step: int


def algorithmic_bytes_per_step(sim) -> int:
    """Each state array read once and written once per step: er, et, hr, ht,
    plasma currents and surface-impedance memory (coefficient tables are
    altitude rows and are not counted)."""

    item = sim.backend.itemsize
    n = sum(int(getattr(sim, f).numel()) for f in ("er", "et", "hr", "ht"))
    if sim._plasma_coupler is not None:
        n += sum(int(j.numel()) for j in sim._plasma_coupler.ade.current_density)
    if sim._surface_impedance_ade is not None:
        n += int(sim._surface_impedance_ade.memory.numel())
    return 2 * item * n


def config1(device: str = "cuda", dtype: str = "float32", seed: int = 20260801, subdivision: int = 2, radial_cells: int = 24, receivers: int = 8, **kwargs) -> Workload:
    from .mesh import build_geodesic_mesh
    from .solver import GeodesicFDTD, SimulationConfig

    cfg = SimulationConfig(subdivision=subdivision, radial_cells=radial_cells)
    mesh = build_geodesic_mesh(subdivision)
    lat, lon = vertex_lat_lon(mesh.vertices, int(np.random.default_rng(seed).integers(mesh.n_vertices)))
    source = GaussianCurrent(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0, carrier_frequency_hz=20.0)
    sim = GeodesicFDTD(cfg, material=ProfileMaterial(), source=source, mesh=mesh, device=device, dtype=dtype, **kwargs)
    rec = uniform_receivers(sim, receivers, seed)
    return Workload("config1", sim, rec, mesh.n_vertices * radial_cells, algorithmic_bytes_per_step(sim))


def config2(device: str = "cuda", dtype: str = "float32", seed: int = 20260805, subdivision: int = 7, radial_cells: int = 40, receivers: int = 64, **kwargs) -> Workload:
    from .mesh import build_geodesic_mesh
    from .solver import GeodesicFDTD, SimulationConfig

    cfg = SimulationConfig(subdivision=subdivision, radial_cells=radial_cells)
    mesh = build_geodesic_mesh(subdivision)
    alt = np.linspace(cfg.minimum_altitude_m, cfg.maximum_altitude_m, cfg.radial_cells + 1)
    mids = 0.5 * (alt[:-1] + alt[1:])
    lat, lon = vertex_lat_lon(mesh.vertices, int(np.random.default_rng(seed).integers(mesh.n_vertices)))
    source = GaussianCurrent(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0, carrier_frequency_hz=50.0)
    sim = GeodesicFDTD(cfg, material=ProfileMaterial(), source=source, plasma=drude_profile_plasma(mesh, mids), mesh=mesh, device=device, dtype=dtype, **kwargs)
    rec = uniform_receivers(sim, receivers, seed)
    return Workload("config2", sim, rec, mesh.n_vertices * radial_cells, algorithmic_bytes_per_step(sim))


def config4(device: str = "cuda", dtype: str = "float32", seed: int = 20260814, subdivision: int = 9, radial_cells: int = 80, receivers: int = 256, **kwargs) -> Workload:
    from .mesh import build_geodesic_mesh
    from .solver import GeodesicFDTD, SimulationConfig
    from .surface_impedance import ConductiveHalfSpaceSurface

    cfg = SimulationConfig(
        subdivision=subdivision, radial_cells=radial_cells, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0,
        radial_boundary_condition="surface-impedance",
    )
    mesh = build_geodesic_mesh(subdivision)
    alt = np.linspace(cfg.minimum_altitude_m, cfg.maximum_altitude_m, cfg.radial_cells + 1)
    mids = 0.5 * (alt[:-1] + alt[1:])
    lat, lon = vertex_lat_lon(mesh.vertices, int(np.random.default_rng(seed).integers(mesh.n_vertices)))
    source = GaussianCurrent(latitude_deg=lat, longitude_deg=lon, altitude_m=2_500.0, peak_current_a=1.0, carrier_frequency_hz=20.0)
    surface = ConductiveHalfSpaceSurface(smooth_log_normal(mesh.edge_midpoints(), seed))
    sim = GeodesicFDTD(
        cfg, material=ProfileMaterial(), source=source, surface_impedance=surface, plasma=drude_profile_plasma(mesh, mids),
        mesh=mesh, device=device, dtype=dtype, **kwargs,
    )
    rec = uniform_receivers(sim, receivers, seed)
    return Workload("config4", sim, rec, mesh.n_vertices * radial_cells, algorithmic_bytes_per_step(sim))


def config3_draws(seed: int = 20260803, members: int = 64) -> list[dict]:
    """The seeded per-member parameters of the ensemble configuration."""

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


def config3_members(device: str = "cuda", dtype: str = "float32", seed: int = 20260803, members: int = 64, receivers: int = 16, **kwargs) -> list[Workload]:
    """The ensemble configuration: ``members`` seeded runs of uneven size and
    physics (one mesh per subdivision level, shared by its members)."""

    from .constants import EPSILON_0
    from .materials import EarthIonosphereMaterial
    from .mesh import build_geodesic_mesh
    from .solver import GeodesicFDTD, SimulationConfig

    meshes: dict[int, object] = {}
    out = []
    for i, d in enumerate(config3_draws(seed, members)):
        sub, L, ground, h0, zeta, sigma0, carrier = (d[k] for k in ("subdivision", "radial_cells", "ground", "h0", "zeta", "sigma0", "carrier"))
        src_draw, rec_seed = d["source_draw"], d["receiver_seed"]
        mesh = meshes.get(sub)
        if mesh is None:
            mesh = meshes[sub] = build_geodesic_mesh(sub)
        material = EarthIonosphereMaterial(
            lithosphere_conductivity_s_m=ground,
            ionosphere_reference_height_m=h0,
            ionosphere_scale_height_m=zeta,
            ionosphere_prefactor_hz=sigma0 / EPSILON_0,
        )
        lat, lon = vertex_lat_lon(mesh.vertices, src_draw % mesh.n_vertices)
        source = GaussianCurrent(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0, carrier_frequency_hz=carrier)
        sim = GeodesicFDTD(SimulationConfig(subdivision=sub, radial_cells=L), material=material, source=source, mesh=mesh,
                           device=device, dtype=dtype, **kwargs)
        rec = uniform_receivers(sim, receivers, rec_seed)
        out.append(Workload(f"config3[{i}]", sim, rec, mesh.n_vertices * L, algorithmic_bytes_per_step(sim)))
    return out


def seed_fields(sim, seed: int = 20260814, amplitude: float = 1.0e-6) -> None:
    """Random initial fields, as the reference benchmark seeds them
    (benchmarks/backend_matrix.py:179-183), generated on the device."""

    torch = sim.backend.torch
    g = torch.Generator(device=sim.backend.torch_device)
    g.manual_seed(seed)
    for f in ("er", "et", "hr", "ht"):
        t = getattr(sim, f)
        # drawn in float64 and rounded, so float32 and float64 runs start from the same state
        t.copy_((torch.randn(t.shape, generator=g, device=t.device, dtype=torch.float64) * amplitude).to(t.dtype))
