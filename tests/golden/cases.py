"""Parity cases shared by the golden-fixture generator and the tests.

Each case is a plain parameter dictionary, so the same inputs can be handed
to the reference (``make_golden.py``, in the build container), to the CPU
oracle and to the CUDA engine.  Materials used by the cases are defined here
as small duck-typed ``sample()`` objects, as the reference's own tests do.
"""

from __future__ import annotations

import numpy as np

EPSILON_0 = 8.854_187_812_8e-12


class ProfileMaterial:
    """Ground sigma/eps below 0 m; air sigma = 0 below ``cutoff_m`` and
    ``min(prefactor * exp((h - h0) / zeta), cap)`` above it."""

    def __init__(
        self,
        ground_sigma=1.0e-2,
        ground_eps=10.0,
        cutoff_m=50_000.0,
        prefactor=1.0e-7,
        h0_m=60_000.0,
        zeta_m=4_000.0,
        cap=1.0e-3,
    ):
        self.ground_sigma = ground_sigma
        self.ground_eps = ground_eps
        self.cutoff_m = cutoff_m
        self.prefactor = prefactor
        self.h0_m = h0_m
        self.zeta_m = zeta_m
        self.cap = cap

    def sample(self, directions, altitudes_m, earth_radius_m):
        h = np.asarray(altitudes_m, dtype=np.float64)
        air = np.minimum(self.prefactor * np.exp((h - self.h0_m) / self.zeta_m), self.cap)
        air = np.where(h < self.cutoff_m, 0.0, air)
        sigma = np.where(h < 0.0, self.ground_sigma, air)
        eps = np.where(h < 0.0, self.ground_eps, 1.0)
        n = len(directions)
        return np.broadcast_to(sigma, (n, len(h))).copy(), np.broadcast_to(eps, (n, len(h))).copy()


class PatchyMaterial:
    """Horizontally varying conductivity (exercises full coefficient arrays)."""

    def sample(self, directions, altitudes_m, earth_radius_m):
        d = np.asarray(directions, dtype=np.float64)
        h = np.asarray(altitudes_m, dtype=np.float64)
        scale = 1.0 + 0.5 * d[:, 2:3] + 0.25 * d[:, 0:1]
        base = np.where(h < 0.0, 2.0e-3, 1.0e-9 * np.exp(h / 20_000.0))
        sigma = scale * base[None, :]
        eps = np.where(h < 0.0, 4.0 + d[:, 1:2] ** 2, np.ones((1, len(h))))
        return sigma, np.broadcast_to(eps, sigma.shape).copy()


def smooth_log_normal(directions, seed: int, median: float = 1.0e-2, spread: float = 0.5):
    """Seeded smooth random field on the sphere: a Gaussian-weighted sum of
    monomials of degree <= 3 in (x, y, z), exponentiated to a log-normal
    map around ``median``."""

    d = np.asarray(directions, dtype=np.float64)
    rng = np.random.default_rng(seed)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    basis = np.stack(
        [x, y, z, x * y, y * z, z * x, x * x - y * y, 3 * z * z - 1, x * y * z, x**3 - 3 * x * y * y, z**3],
        axis=1,
    )
    field = basis @ rng.standard_normal(basis.shape[1])
    field = (field - field.mean()) / max(field.std(), 1e-30)
    return median * np.exp(spread * field)


def profile_plasma_arrays(n_faces: int, midpoint_altitudes_m, magnetic_t: float = 0.0):
    """Electron density n_e(h)=1e6 exp((h-85 km)/3 km) and collision frequency
    nu(h)=1e7 exp(-(h-70 km)/6 km) on faces x midpoints; B along +z."""

    h = np.asarray(midpoint_altitudes_m, dtype=np.float64)
    density = np.broadcast_to(1.0e6 * np.exp((h - 85_000.0) / 3_000.0), (n_faces, len(h))).copy()
    collision = np.broadcast_to(1.0e7 * np.exp(-(h - 70_000.0) / 6_000.0), (n_faces, len(h))).copy()
    magnetic = np.zeros((n_faces, len(h), 3))
    magnetic[..., 2] = magnetic_t
    return magnetic, density, collision


def vertex_lat_lon(vertices, index: int) -> tuple[float, float]:
    v = np.asarray(vertices)[index]
    return float(np.degrees(np.arcsin(np.clip(v[2], -1.0, 1.0)))), float(np.degrees(np.arctan2(v[1], v[0])))


# ---------------------------------------------------------------------------
# Case table.  "init" seeds 1e-6 * N(0, 1) fields (or the given amplitude);
# "material" is one of: "default" (EarthIonosphereMaterial()), "profile",
# "patchy", ("earth", {params}).
# ---------------------------------------------------------------------------

CASES: dict[str, dict] = {
    "random_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.2),
        material="default",
        init=(20260805, 1.0e-6),
        steps=5,
    ),
    "source_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.2),
        material="default",
        source=dict(kind="vertical", peak_current_a=1.0e6),
        steps=40,
    ),
    "nonuniform_s0": dict(
        config=dict(
            subdivision=0,
            radial_cells=5,
            minimum_altitude_m=-10_000.0,
            maximum_altitude_m=4_000.0,
            radial_altitudes_m=(-10_000.0, -6_000.0, -2_000.0, -1_000.0, 0.0, 4_000.0),
            radial_grid_policy="allow-abrupt",
            courant_factor=0.2,
        ),
        material="default",
        init=(20260805, 1.0e-6),
        steps=5,
    ),
    "thin_shell_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.25, geometry_mode="thin-shell"),
        material="patchy",
        init=(42, 1.0e-6),
        steps=6,
    ),
    "trapezoidal_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.25, loss_integration="trapezoidal"),
        material=("earth", dict(lithosphere_conductivity_s_m=1.0e-2)),
        init=(20260814, 1.0e-6),
        steps=6,
    ),
    "tangential_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.25),
        material="default",
        source=dict(kind="tangential", peak_current_a=1.0e6, azimuths_deg=(30.0, 120.0), line_lengths_m=(2.0, 3.0), altitude_m=0.0),
        steps=20,
    ),
    "surface_s1": dict(
        config=dict(
            subdivision=1,
            radial_cells=4,
            minimum_altitude_m=0.0,
            maximum_altitude_m=100_000.0,
            courant_factor=0.2,
            radial_boundary_condition="surface-impedance",
        ),
        material="default",
        surface=dict(conductivity="scalar", value=1.0 / 50.0),
        init=(20260820, 1.0e-9),
        steps=4,
    ),
    "surface_map_s2": dict(
        config=dict(
            subdivision=2,
            radial_cells=6,
            minimum_altitude_m=0.0,
            maximum_altitude_m=100_000.0,
            courant_factor=0.3,
            radial_boundary_condition="surface-impedance",
        ),
        material="profile",
        surface=dict(conductivity="smooth", seed=7),
        init=(20260820, 1.0e-9),
        steps=12,
    ),
    "plasma_magnetized_s0": dict(
        config=dict(subdivision=0, radial_cells=2, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.2),
        material="default",
        plasma=dict(kind="uniform", magnetic_t=50.0e-6, density_m3=1.0e4, collision_hz=200.0),
        init=(20260820, 1.0e-9),
        steps=3,
    ),
    "plasma_magnetized_s1": dict(
        config=dict(subdivision=1, radial_cells=5, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.25),
        material="default",
        plasma=dict(kind="uniform", magnetic_t=40.0e-6, density_m3=1.0e6, collision_hz=1.0e4, two_species=True),
        init=(11, 1.0e-9),
        steps=6,
    ),
    "plasma_drude_s2": dict(
        config=dict(subdivision=2, radial_cells=10, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.35),
        material="profile",
        plasma=dict(kind="profile", magnetic_t=0.0),
        source=dict(kind="vertical", peak_current_a=1.0, carrier_frequency_hz=50.0, center_time_s=2.0e-4, one_over_e_half_width_s=1.0e-4, seed_vertex=3),
        init=(5, 1.0e-9),
        steps=60,
    ),
    "config4_mini_s2": dict(
        config=dict(
            subdivision=2,
            radial_cells=8,
            minimum_altitude_m=0.0,
            maximum_altitude_m=100_000.0,
            courant_factor=0.35,
            radial_boundary_condition="surface-impedance",
        ),
        material="profile",
        surface=dict(conductivity="smooth", seed=20260814),
        plasma=dict(kind="profile", magnetic_t=0.0),
        source=dict(kind="vertical", peak_current_a=1.0, carrier_frequency_hz=20.0, center_time_s=3.0e-4, one_over_e_half_width_s=1.5e-4, seed_vertex=17),
        receivers=dict(seed=20260814, count=12),
        steps=50,
    ),
    "config1_s2": dict(
        config=dict(subdivision=2, radial_cells=24, earth_radius_m=6_370_000.0, courant_factor=0.35),
        material="profile",
        source=dict(kind="vertical", peak_current_a=1.0, carrier_frequency_hz=20.0, seed_vertex=20260805),
        receivers=dict(seed=20260805, count=8),
        steps=1000,
    ),
    # locally refined meshes (adaptive_mesh.py): base level, refinement regions
    # (lat, lon, radius, target level, transition width, label); vertex degree 7-8
    "adaptive_s1": dict(
        config=dict(subdivision=1, radial_cells=6, courant_factor=0.2),
        adaptive=(1, ((35.0, 126.0, 8.0, 3, 8.0, "source"),)),
        material="default",
        source=dict(kind="vertical", peak_current_a=1.0e6, seed_vertex=20260806),
        init=(20260807, 1.0e-6),
        steps=12,
    ),
    "adaptive_plasma_si_s1": dict(
        config=dict(subdivision=1, radial_cells=5, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.25,
                    radial_boundary_condition="surface-impedance"),
        adaptive=(1, ((46.5, -90.9, 8.0, 3, 8.0, "source"), (69.0, -156.0, 8.0, 3, 8.0, "oil"))),
        material="default",
        surface=dict(conductivity="scalar", value=1.0e-2),
        plasma=dict(kind="uniform", magnetic_t=40.0e-6, density_m3=1.0e6, collision_hz=1.0e4, two_species=True),
        init=(13, 1.0e-9),
        steps=8,
    ),
}


def receiver_rows(n_vertices: int, altitudes_m, seed: int, count: int):
    """Seed-chosen distinct surface vertices, node nearest 0 m, weight 1."""

    rng = np.random.default_rng(seed)
    vertices = rng.choice(n_vertices, size=count, replace=False).astype(np.int64)
    layer = int(np.argmin(np.abs(np.asarray(altitudes_m) - 0.0)))
    return vertices[:, None], np.full(count, layer, dtype=np.int64), np.ones((count, 1))


def source_vertex(n_vertices: int, seed: int) -> int:
    return int(np.random.default_rng(seed).integers(n_vertices))


def initial_fields(shapes: dict[str, tuple[int, ...]], seed: int, amplitude: float) -> dict[str, np.ndarray]:
    """Seeded N(0,1) * amplitude fields in er, et, hr, ht order."""

    rng = np.random.default_rng(seed)
    return {name: amplitude * rng.standard_normal(shapes[name]) for name in ("er", "et", "hr", "ht")}


# record_receiver_traces fixture (visualization.py:212-252): receivers as
# (latitude, longitude, altitude, label), 11 steps sampled every 4 (rows at 0, 4, 8, 11)
RECEIVER_TRACES = dict(
    case="source_s1",
    steps=11,
    sample_every=4,
    receivers=(
        (35.1595, 126.8526, 0.0, "gwangju"),
        (-12.5, 40.0, 30_000.0, None),
        (89.0, -170.0, 95_000.0, "polar"),
    ),
)


# build_refined_radial_grid fixtures (radial_grid.py:44-132): (minimum, maximum,
# background step, ((region minimum, region maximum, region step), ...))
RADIAL_GRIDS = (
    (0.0, 100_000.0, 10_000.0, ((60_000.0, 90_000.0, 1_000.0),)),
    (0.0, 100_000.0, 10_000.0, ((40_000.0, 80_000.0, 2_000.0), (60_000.0, 70_000.0, 500.0))),
    (-100_000.0, 100_000.0, 7_000.0, ((-3_000.0, 4_000.0, 150.0), (55_000.0, 99_000.0, 900.0))),
    (0.0, 90_000.0, 3_333.0, ((0.0, 1_000.0, 37.0),)),
    (-5_000.0, 5_000.0, 2_500.0, ()),
)
