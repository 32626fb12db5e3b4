"""``SimulationConfig`` and ``GeodesicFDTD`` with the reference's public API.

Drop-in for the reference's ``GeodesicFDTD`` on its PyTorch CUDA backend
(src/ionosphere_fdtd/solver.py:30-1294): same constructor, attributes,
validation messages, ``step()``, observation recording, ``diagnostics()`` and
checkpoint layout.  The host does exactly the reference's setup (material
sampling, CFL limit, loss coefficients, source supports, ADE coefficients)
and hands it to a native plan; every time step then runs as two fused CUDA
launches (H phase, E phase) on torch's current stream, replayed from CUDA
graphs in chunks.  There is no CPU fallback: without a CUDA device the
constructor raises ``BackendUnavailableError``.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .backend import CudaBackend, create_backend
from .constants import C_0, EARTH_RADIUS_M, EPSILON_0, MU_0
from ._native import row_pitch
from .engine import Engine, Physics, Tuning, plasma_inputs, surface_inputs
from .materials import EarthIonosphereMaterial
from .mesh import GeodesicMesh, build_geodesic_mesh
from .plasma import GeodesicPlasmaCoupler, MeshPlasmaModel
from .provenance import distinct_elements
from .radial_grid import validate_radial_grid
from .sources import GaussianCurrent, TangentialGaussianCurrent
from .surface_impedance import ConductiveHalfSpaceSurface, SurfaceImpedanceADE


@dataclass(frozen=True, slots=True)
class SimulationConfig:
    """Geometry and integration controls (solver.py:30-171)."""

    subdivision: int = 2
    radial_cells: int = 24
    minimum_altitude_m: float = -100_000.0
    maximum_altitude_m: float = 100_000.0
    earth_radius_m: float = EARTH_RADIUS_M
    courant_factor: float = 0.35
    time_step_s: float | None = None
    mesh_relaxations: int = 0
    mesh_optimization_steps: int = 0
    mesh_orientation: str = "polar"
    radial_altitudes_m: tuple[float, ...] | None = None
    radial_material_support: str = "point"
    tangential_material_support: str = "point"
    horizontal_anomaly_mode: str = "point"
    radial_boundary_condition: str = "pec"
    loss_integration: str = "exponential"
    radial_grid_policy: str = "smooth"
    geometry_mode: str = "full-spherical"
    compress_uniform_material_coefficients: bool = False

    def __post_init__(self) -> None:
        integers = (self.subdivision, self.radial_cells, self.mesh_relaxations, self.mesh_optimization_steps)
        if any(isinstance(v, bool) or not isinstance(v, (int, np.integer)) for v in integers):
            raise ValueError("mesh and radial cell controls must be integers")
        if self.subdivision < 0:
            raise ValueError("subdivision must be non-negative")
        if self.radial_cells < 2:
            raise ValueError("radial_cells must be at least 2")
        if self.mesh_relaxations < 0:
            raise ValueError("mesh_relaxations must be non-negative")
        if self.mesh_optimization_steps < 0:
            raise ValueError("mesh_optimization_steps must be non-negative")
        choices = (
            ("mesh_orientation", {"native", "polar"}, "mesh_orientation must be 'native' or 'polar'"),
            ("radial_material_support", {"point", "dual-cell"}, "radial_material_support must be 'point' or 'dual-cell'"),
            ("tangential_material_support", {"point", "edge-diamond"}, "tangential_material_support must be 'point' or 'edge-diamond'"),
            ("horizontal_anomaly_mode", {"point", "conservative-nearest"}, "horizontal_anomaly_mode must be 'point' or 'conservative-nearest'"),
            ("radial_boundary_condition", {"pec", "surface-impedance"}, "radial_boundary_condition must be 'pec' or 'surface-impedance'"),
        )
        for name, allowed, message in choices:
            if getattr(self, name) not in allowed:
                raise ValueError(message)
        if self.radial_boundary_condition == "surface-impedance" and self.minimum_altitude_m != 0.0:
            raise ValueError("surface-impedance boundary requires minimum_altitude_m=0")
        if self.loss_integration not in {"exponential", "trapezoidal"}:
            raise ValueError("loss_integration must be 'exponential' or 'trapezoidal'")
        if self.radial_grid_policy not in {"smooth", "balanced-2to1", "allow-abrupt"}:
            raise ValueError("radial_grid_policy must be 'smooth', 'balanced-2to1', or 'allow-abrupt'")
        if self.geometry_mode not in {"full-spherical", "thin-shell"}:
            raise ValueError("geometry_mode must be 'full-spherical' or 'thin-shell'")
        if not all(np.isfinite(v) for v in (self.minimum_altitude_m, self.maximum_altitude_m, self.earth_radius_m, self.courant_factor)):
            raise ValueError("geometry and Courant controls must be finite")
        if self.minimum_altitude_m >= self.maximum_altitude_m:
            raise ValueError("altitude bounds are reversed")
        if self.earth_radius_m + self.minimum_altitude_m <= 0.0:
            raise ValueError("minimum radius must be positive")
        if not 0.0 < self.courant_factor <= 1.0:
            raise ValueError("courant_factor must be in (0, 1]")
        if self.time_step_s is not None and (not np.isfinite(self.time_step_s) or self.time_step_s <= 0.0):
            raise ValueError("time_step_s must be finite and positive")
        if self.radial_altitudes_m is not None:
            alt = np.asarray(self.radial_altitudes_m, dtype=np.float64)
            if alt.ndim != 1 or len(alt) < 3 or not np.all(np.isfinite(alt)) or not np.all(np.diff(alt) > 0.0):
                raise ValueError("radial_altitudes_m must contain at least three finite, increasing values")
            if len(alt) != self.radial_cells + 1:
                raise ValueError("radial_cells must equal len(radial_altitudes_m) - 1")
            if alt[0] != self.minimum_altitude_m or alt[-1] != self.maximum_altitude_m:
                raise ValueError("custom radial altitudes must include the configured altitude bounds")
            steps = np.diff(alt)
            change = self.radial_cells * np.abs(np.diff(steps)) / np.minimum(steps[:-1], steps[1:])
            if self.radial_grid_policy == "smooth" and np.any(change > 8.0 * (1.0 + 1.0e-12)):
                raise ValueError(
                    "custom radial grid is not smoothly graded; use a smooth node "
                    "mapping or explicitly select radial_grid_policy='allow-abrupt'"
                )
            if self.radial_grid_policy == "balanced-2to1":
                validate_radial_grid(alt, maximum_adjacent_step_ratio=2.0)


def _validated_material_sample(values, expected_shape, label):
    """solver.py:763-787."""

    try:
        sigma_values, epsilon_values = values
    except (TypeError, ValueError) as error:
        raise ValueError(f"{label} material sampler must return conductivity and permittivity") from error
    sigma = np.asarray(sigma_values, dtype=np.float64)
    eps = np.asarray(epsilon_values, dtype=np.float64)
    if sigma.shape != expected_shape or eps.shape != expected_shape:
        raise ValueError(f"{label} material arrays must have shape {expected_shape}")
    # every element is checked once: a broadcast (zero-stride) axis repeats the same values
    s_core, e_core = distinct_elements(sigma), distinct_elements(eps)
    if not np.all(np.isfinite(s_core)) or not np.all(np.isfinite(e_core)):
        raise ValueError(f"{label} material arrays must be finite")
    if np.any(s_core < 0.0):
        raise ValueError(f"{label} conductivity cannot be negative")
    if np.any(e_core <= 0.0):
        raise ValueError(f"{label} relative permittivity must be positive")
    return sigma, eps


def _uniform_rows(values: NDArray[np.float64]) -> bool:
    a = np.asarray(values)
    if a.shape[0] <= 1 or a.strides[0] == 0:
        return True
    return bool(np.array_equal(a, np.broadcast_to(a[:1], a.shape)))


class GeodesicFDTD:
    """Earth-ionosphere FDTD on staggered geodesic radial planes.

    ``er``/``ht`` live on radial nodes (TM-r), ``hr``/``et`` on midpoints
    (TE-r); H is staggered half a step behind E (solver.py:174-182).
    """

    def __init__(
        self,
        config: SimulationConfig | None = None,
        material: Any = None,
        source: GaussianCurrent | TangentialGaussianCurrent | None = None,
        surface_impedance: ConductiveHalfSpaceSurface | None = None,
        plasma: MeshPlasmaModel | None = None,
        mesh: GeodesicMesh | None = None,
        backend: str = "torch",
        device: str = "auto",
        dtype: str = "auto",
        compile_step: bool = False,
        compile_chunk_size: int = 8,
        torch_threads: int | None = None,
        *,
        tuning: Tuning | None = None,
    ) -> None:
        if isinstance(compile_chunk_size, bool) or not isinstance(compile_chunk_size, (int, np.integer)) or compile_chunk_size < 1:
            raise ValueError("compile_chunk_size must be a positive integer")
        self.compile_chunk_size = int(compile_chunk_size)
        self.config = config or SimulationConfig()
        if mesh is None:
            self.mesh = build_geodesic_mesh(
                subdivision=self.config.subdivision,
                relaxations=self.config.mesh_relaxations,
                orientation=self.config.mesh_orientation,
                optimization_steps=self.config.mesh_optimization_steps,
            )
        else:
            if self.config.mesh_relaxations or self.config.mesh_optimization_steps:
                raise ValueError("mesh relaxation and optimization controls cannot accompany a provided mesh")
            if mesh.topology_kind == "uniform":
                polar = np.count_nonzero(
                    (mesh.vertex_degree == 5) & np.isclose(np.abs(mesh.vertices[:, 2]), 1.0, rtol=0.0, atol=1.0e-13)
                )
                if polar != (2 if self.config.mesh_orientation == "polar" else 0):
                    raise ValueError("provided mesh orientation does not match config")
            self.mesh = mesh
        if self.mesh.subdivision is not None and self.mesh.subdivision != self.config.subdivision:
            raise ValueError("provided mesh subdivision does not match config")
        self.backend: CudaBackend = create_backend(backend, self.mesh, device=device, dtype=dtype, torch_threads=torch_threads)
        self.material = material or EarthIonosphereMaterial()
        self.source = source
        self.surface_impedance = surface_impedance
        self.plasma = plasma
        if self.config.radial_boundary_condition == "surface-impedance":
            if surface_impedance is None:
                raise ValueError("surface-impedance boundary requires a surface model")
        elif surface_impedance is not None:
            raise ValueError("surface impedance model requires radial_boundary_condition='surface-impedance'")

        cfg = self.config
        if cfg.radial_altitudes_m is None:
            self.altitudes_m = np.linspace(cfg.minimum_altitude_m, cfg.maximum_altitude_m, cfg.radial_cells + 1)
        else:
            self.altitudes_m = np.asarray(cfg.radial_altitudes_m, dtype=np.float64)
        self.radii_m = cfg.earth_radius_m + self.altitudes_m
        self.radial_midpoints_m = 0.5 * (self.radii_m[:-1] + self.radii_m[1:])
        self.radial_midpoint_altitudes_m = self.radial_midpoints_m - cfg.earth_radius_m
        self.radial_steps_m = np.diff(self.radii_m)
        ctrl = np.empty(len(self.radii_m), dtype=np.float64)
        ctrl[0] = 0.5 * self.radial_steps_m[0]
        ctrl[-1] = 0.5 * self.radial_steps_m[-1]
        ctrl[1:-1] = np.diff(self.radial_midpoints_m)
        self.radial_node_control_lengths_m = ctrl
        if plasma is not None:
            plasma.validate_grid(self.mesh, self.radial_midpoint_altitudes_m)

        self._sample_material_properties()
        self.cfl_time_step_limit_s = self._estimate_cfl_time_step_limit()
        self.maximum_stable_time_step_s = cfg.courant_factor * self.cfl_time_step_limit_s
        self.time_step_s = cfg.time_step_s if cfg.time_step_s is not None else self.maximum_stable_time_step_s
        if self.time_step_s > self.maximum_stable_time_step_s * (1.0 + 1.0e-12):
            raise ValueError(
                f"time step {self.time_step_s:.6e} s exceeds conservative limit {self.maximum_stable_time_step_s:.6e} s"
            )
        if self.source is not None and self.source.carrier_frequency_hz >= 0.5 / self.time_step_s:
            raise ValueError("source carrier frequency must be below the time-step Nyquist limit")

        b = self.backend
        L = len(self.radial_midpoints_m)
        self._node_pitch, self._mid_pitch = row_pitch(L + 1), row_pitch(L)
        # padded, 16-byte aligned rows for the step kernels; the public fields
        # are exact-shape views (padding stays zero)
        self._buffers = {
            "er": b.zeros((self.mesh.n_vertices, self._node_pitch)),
            "et": b.zeros((self.mesh.n_edges, self._mid_pitch)),
            "hr": b.zeros((self.mesh.n_faces, self._mid_pitch)),
            "ht": b.zeros((self.mesh.n_edges, self._node_pitch)),
        }
        self._views = {
            "er": self._buffers["er"][:, : L + 1],
            "et": self._buffers["et"][:, :L],
            "hr": self._buffers["hr"][:, :L],
            "ht": self._buffers["ht"][:, : L + 1],
        }
        self._surface_impedance_ade = (
            SurfaceImpedanceADE(surface_impedance, edge_count=self.mesh.n_edges, time_step_s=self.time_step_s, backend=b)
            if surface_impedance is not None
            else None
        )
        self._plasma_coupler = (
            GeodesicPlasmaCoupler(plasma, self.mesh, self.radial_midpoint_altitudes_m, self.time_step_s, b, self._mid_pitch)
            if plasma is not None
            else None
        )
        self._prepare_geometry()
        self._prepare_material_coefficients()
        self._source_distribution = None
        self._tangential_source_distribution = None
        if isinstance(self.source, TangentialGaussianCurrent):
            self._tangential_source_distribution = self.source.edge_distribution(self)
        elif self.source is not None:
            self._source_distribution = self.source.staggered_distribution(self)
        self.time_s = 0.0
        self.steps = 0
        self.compiled = bool(compile_step)
        if tuning is None:
            tuning = Tuning(graph_chunk=max(self.compile_chunk_size, 8) if compile_step else 32)
        self._engine = Engine(
            self.mesh, self.radii_m, cfg.geometry_mode == "full-spherical", self.time_step_s, self._physics(), b, tuning
        )
        if (self._engine.node_pitch, self._engine.mid_pitch) != (self._node_pitch, self._mid_pitch):
            raise RuntimeError("native plan chose a different row pitch than the host layout")
        b._engine = self._engine

    # -- fields: exact-shape views of padded device buffers -----------------------

    def _assign_field(self, name: str, value: Any) -> None:
        view = self._views[name]
        torch = self.backend.torch
        t = value if torch.is_tensor(value) else torch.as_tensor(np.asarray(value))
        if tuple(t.shape) != tuple(view.shape):
            raise ValueError(f"{name} must have shape {tuple(view.shape)}, got {tuple(t.shape)}")
        if t.data_ptr() != view.data_ptr():
            view.copy_(t.to(device=view.device, dtype=view.dtype))

    er = property(lambda self: self._views["er"], lambda self, v: self._assign_field("er", v))
    et = property(lambda self: self._views["et"], lambda self, v: self._assign_field("et", v))
    hr = property(lambda self: self._views["hr"], lambda self, v: self._assign_field("hr", v))
    ht = property(lambda self: self._views["ht"], lambda self, v: self._assign_field("ht", v))

    # -- setup (host, float64) ----------------------------------------------------

    def _estimate_cfl_time_step_limit(self) -> float:
        """solver.py:377-406."""

        r0 = float(self.radii_m.min())
        primal = r0 * float(self.mesh.primal_edge_angles.min())
        dual = r0 * float(self.mesh.dual_edge_angles.min())
        radial = float(self.radial_steps_m.min())
        inverse_length_squared = primal**-2 + dual**-2 + (2.0 / radial) ** 2
        eps_min = min(float(np.min(self.epsilon_r_er)), float(np.min(self.epsilon_r_et)))
        limit = np.sqrt(eps_min) / (C_0 * np.sqrt(inverse_length_squared))
        if self.plasma is None:
            return float(limit)
        densities = [s.number_density_m3 for s in self.plasma.species]
        rows = (lambda a: a[:1]) if all(_uniform_rows(a) for a in densities) else (lambda a: a)
        drive = np.zeros(rows(self.plasma.magnetic_field_t[..., 0]).shape)
        for s in self.plasma.species:
            drive = drive + rows(s.number_density_m3) * s.charge_c**2 / s.mass_kg
        wp = np.sqrt(float(np.max(drive)) / (EPSILON_0 * eps_min))
        if wp == 0.0:
            return float(limit)
        return float(min(limit, 2.0 / wp))

    def _sample_material_properties(self) -> None:
        """Point-support material sampling (solver.py:467-629).

        Mesh-native samplers (``sample_mesh``) are honoured; the reference's
        dual-cell / edge-diamond quadrature supports and conservative anomaly
        fractions are host-side material preprocessing that this build does not
        reproduce, and selecting them raises ``ValueError``.
        """

        cfg = self.config
        sampler = getattr(self.material, "sample_mesh", None)
        if sampler is not None:
            values = sampler(
                self.mesh,
                self.altitudes_m,
                cfg.earth_radius_m,
                radial_material_support=cfg.radial_material_support,
                tangential_material_support=cfg.tangential_material_support,
                horizontal_anomaly_mode=cfg.horizontal_anomaly_mode,
            )
            try:
                sigma_er, eps_er, sigma_et, eps_et = values
            except (TypeError, ValueError) as error:
                raise ValueError("mesh material sampler must return four property arrays") from error
            self.sigma_er, self.epsilon_r_er = _validated_material_sample(
                (sigma_er, eps_er), (self.mesh.n_vertices, len(self.altitudes_m)), "mesh-native radial"
            )
            self.sigma_et, self.epsilon_r_et = _validated_material_sample(
                (sigma_et, eps_et), (self.mesh.n_edges, len(self.radial_midpoint_altitudes_m)), "mesh-native tangential"
            )
            return
        if cfg.radial_material_support != "point" or cfg.tangential_material_support != "point" or cfg.horizontal_anomaly_mode != "point":
            raise ValueError(
                "only point material support is implemented by this engine; sample the material with a "
                "mesh-native sampler (sample_mesh) for quadrature supports"
            )
        self.sigma_er, self.epsilon_r_er = _validated_material_sample(
            self.material.sample(self.mesh.vertices, self.altitudes_m, cfg.earth_radius_m),
            (self.mesh.n_vertices, len(self.altitudes_m)),
            "radial",
        )
        sample_cells = getattr(self.material, "sample_tangential_cells", None)
        midpoints = self.mesh.edge_midpoints()
        values = (
            self.material.sample(midpoints, self.radial_midpoint_altitudes_m, cfg.earth_radius_m)
            if sample_cells is None
            else sample_cells(midpoints, self.altitudes_m[:-1], self.altitudes_m[1:], cfg.earth_radius_m)
        )
        self.sigma_et, self.epsilon_r_et = _validated_material_sample(
            values, (self.mesh.n_edges, len(self.radial_midpoint_altitudes_m)), "tangential"
        )

    def _prepare_geometry(self) -> None:
        """Per-entity and per-layer metric factors (solver.py:408-442), kept on the device
        for API parity; the step kernels read their own copies from the plan."""

        b = self.backend
        m = self.mesh
        self._primal_edge_angles = b.asarray(m.primal_edge_angles[:, None])
        self._inverse_primal_edge_angles = b.asarray(1.0 / m.primal_edge_angles[:, None])
        self._dual_edge_angles = b.asarray(m.dual_edge_angles[:, None])
        self._inverse_dual_edge_angles = b.asarray(1.0 / m.dual_edge_angles[:, None])
        self._inverse_dual_cell_solid_angles = b.asarray(1.0 / m.dual_cell_solid_angles[:, None])
        self._inverse_face_solid_angles = b.asarray(1.0 / m.face_solid_angles[:, None])
        self._radii = b.asarray(self.radii_m)
        self._inverse_radii = b.asarray(1.0 / self.radii_m[None, :])
        self._radial_midpoints = b.asarray(self.radial_midpoints_m)
        self._inverse_radial_midpoints = b.asarray(1.0 / self.radial_midpoints_m[None, :])
        self._radial_steps = b.asarray(self.radial_steps_m)
        self._radial_node_control_lengths = b.asarray(self.radial_node_control_lengths_m)
        self._radial_center_distances = b.asarray(self.radial_midpoints_m[1:] - self.radial_midpoints_m[:-1])

    def _loss_rule(self, sigma, epsilon):
        dt = self.time_step_s
        if self.config.loss_integration == "trapezoidal":
            q = sigma * dt / (2.0 * epsilon)
            return (1.0 - q) / (1.0 + q), dt / (epsilon * (1.0 + q))
        rate = sigma * dt / epsilon
        decay = np.exp(-rate)
        phi = np.ones_like(rate)
        nz = rate != 0.0
        phi[nz] = -np.expm1(-rate[nz]) / rate[nz]
        return decay, dt / epsilon * phi

    def _prepare_material_coefficients(self) -> None:
        """Loss coefficients (solver.py:706-761).  Horizontally uniform
        materials keep one altitude row (bitwise the same values)."""

        compress = self.config.compress_uniform_material_coefficients
        uniform = all(_uniform_rows(a) for a in (self.sigma_er, self.epsilon_r_er, self.sigma_et, self.epsilon_r_et))
        if compress and not uniform:
            raise ValueError("cannot compress horizontally varying radial electric coefficients")
        rows = (lambda a: np.asarray(a)[:1]) if uniform else (lambda a: np.asarray(a))
        ca_er, cb_er = self._loss_rule(rows(self.sigma_er), EPSILON_0 * rows(self.epsilon_r_er))
        ca_et, cb_et = self._loss_rule(rows(self.sigma_et), EPSILON_0 * rows(self.epsilon_r_et))
        self._coef_host = tuple(np.ascontiguousarray(a, dtype=np.float64) for a in (ca_er, cb_er, ca_et, cb_et))
        b = self.backend
        self._ca_er, self._cb_er, self._ca_et, self._cb_et = (b.asarray(a) for a in self._coef_host)

    def _physics(self) -> Physics:
        ca_er, cb_er, ca_et, cb_et = self._coef_host
        inv_dual_area = 1.0 / self.mesh.dual_cell_solid_angles
        inv_phi = 1.0 / self.mesh.dual_edge_angles
        src_er = src_et = None
        if self._source_distribution is not None:
            v, k, w = (np.asarray(a) for a in self._source_distribution)
            row = v if ca_er.shape[0] > 1 else np.zeros_like(v)
            coef = cb_er[row, k] * w * self.source.vertical_element_length_m * inv_dual_area[v] / self.radii_m[k] ** 2 / self.radial_node_control_lengths_m[k]
            src_er = (v.astype(np.int64), k.astype(np.int64), coef)
        if self._tangential_source_distribution is not None:
            e, j, w = (np.asarray(a) for a in self._tangential_source_distribution)
            row = e if ca_et.shape[0] > 1 else np.zeros_like(e)
            coef = cb_et[row, j] * w * inv_phi[e] / self.radial_midpoints_m[j] / self.radial_steps_m[j]
            src_et = (e.astype(np.int64), j.astype(np.int64), coef)
        full = self.config.geometry_mode == "full-spherical"
        si = surface_inputs(self._surface_impedance_ade, self.radii_m, self.radial_midpoints_m, full) if self._surface_impedance_ade else None
        pl = plasma_inputs(self._plasma_coupler) if self._plasma_coupler else None
        return Physics(ca_er, cb_er, ca_et, cb_et, src_er, src_et, si, pl)

    # -- state binding ------------------------------------------------------------------

    def _state(self):
        ade = self._surface_impedance_ade
        currents = tuple(self._plasma_coupler.ade.buffers) if self._plasma_coupler else ()
        buf = self._buffers
        memory = ade.memory.contiguous() if ade is not None else None
        if ade is not None and memory.data_ptr() != ade.memory.data_ptr():
            ade.memory = memory
        return self._engine.state(buf["er"], buf["et"], buf["hr"], buf["ht"], memory, currents)

    def _source_currents(self, count: int) -> NDArray[np.float64] | None:
        """I((n + 1/2) dt) for the next ``count`` steps, float64 (solver.py:851-865)."""

        if self.source is None:
            return None
        times = (self.steps + np.arange(count, dtype=np.float64) + 0.5) * self.time_step_s
        series = getattr(self.source, "current_series", None)
        if series is not None:
            return np.asarray(series(times, self.time_step_s), dtype=np.float64)
        return np.fromiter((self.source.current_a(float(t), self.time_step_s) for t in times), dtype=np.float64, count=count)

    # -- time stepping ---------------------------------------------------------------

    def step(self, count: int = 1) -> None:
        """Advance ``count`` complete leapfrog steps (solver.py:789-816)."""

        count = self._validated_count(count, "step count", minimum=0)
        if not count:
            return
        self._engine.step(self._state(), self._source_currents(count), count)
        self.steps += count
        self.time_s = self.steps * self.time_step_s

    def _update_magnetic_fields(self) -> None:
        """The H half step alone (solver.py:877-921)."""

        self._engine.update_magnetic(self._state())

    def _update_electric_fields(self, current_a: float = 0.0) -> None:
        """The E half step alone with source current ``current_a`` (solver.py:923-989)."""

        self._engine.update_electric(self._state(), float(current_a))

    def _advance_fields(self, current_a: Any) -> None:
        self._update_magnetic_fields()
        self._update_electric_fields(float(current_a))

    # -- checkpoints -----------------------------------------------------------------

    def save_checkpoint(self, path: str | Path, *, compress: bool = True) -> Path:
        from .checkpoint import save_checkpoint

        return save_checkpoint(self, path, compress=compress)

    @classmethod
    def load_checkpoint(
        cls,
        path: str | Path,
        *,
        backend: str = "torch",
        device: str = "auto",
        dtype: str | None = None,
        compile_step: bool = False,
        compile_chunk_size: int = 8,
        torch_threads: int | None = None,
    ) -> "GeodesicFDTD":
        from .checkpoint import load_checkpoint

        return load_checkpoint(
            path,
            backend=backend,
            device=device,
            dtype=dtype,
            compile_step=compile_step,
            compile_chunk_size=compile_chunk_size,
            torch_threads=torch_threads,
        )

    # -- diagnostics -----------------------------------------------------------------

    def diagnostics(self) -> dict[str, float | int | str]:
        """Scalar diagnostics (solver.py:991-1031); the four maxima come from one
        reduction launch and one device-to-host copy."""

        maxima = self._engine.max_abs(self._state())
        return {
            "step": self.steps,
            "time_s": self.time_s,
            "electric_time_s": self.electric_time_s,
            "magnetic_time_s": self.magnetic_time_s,
            "backend": self.backend.name,
            "device": self.backend.device,
            "dtype": self.backend.dtype_name,
            "compiled": self.compiled,
            "compile_chunk_size": self.compile_chunk_size,
            "radial_boundary_condition": self.config.radial_boundary_condition,
            "surface_impedance_terms": self.surface_impedance.terms if self.surface_impedance is not None else 0,
            "surface_impedance_state_bytes": self._surface_impedance_ade.state_bytes if self._surface_impedance_ade else 0,
            "plasma_species": len(self.plasma.species) if self.plasma else 0,
            "plasma_state_bytes": self._plasma_coupler.ade.state_bytes if self._plasma_coupler else 0,
            "loss_integration": self.config.loss_integration,
            "geometry_mode": self.config.geometry_mode,
            "cfl_time_step_limit_s": self.cfl_time_step_limit_s,
            "courant_factor": self.config.courant_factor,
            "field_memory_bytes": self.memory_bytes,
            "persistent_backend_bytes": self.persistent_backend_bytes,
            "max_abs_er_v_m": float(maxima[0]),
            "max_abs_et_v_m": float(maxima[1]),
            "max_abs_hr_a_m": float(maxima[2]),
            "max_abs_ht_a_m": float(maxima[3]),
        }

    @property
    def electric_time_s(self) -> float:
        return self.steps * self.time_step_s

    @property
    def magnetic_time_s(self) -> float:
        return (self.steps - 0.5) * self.time_step_s

    def to_numpy(self, values: Any) -> NDArray[np.generic]:
        return self.backend.to_numpy(values)

    def field_value(self, field: str, *indices: int) -> float:
        if field not in {"er", "et", "hr", "ht"}:
            raise ValueError("field must be er, et, hr, or ht")
        return self.backend.scalar(getattr(self, field)[indices])

    @staticmethod
    def _validated_count(value: int, label: str, *, minimum: int) -> int:
        if isinstance(value, bool) or not isinstance(value, (int, np.integer)):
            raise ValueError(f"{label} must be an integer")
        result = int(value)
        if result < minimum:
            raise ValueError(f"{label} must be {'non-negative' if minimum == 0 else 'positive'}")
        return result

    @staticmethod
    def _validated_index_array(values: Any, label: str) -> NDArray[np.int64]:
        array = np.asarray(values)
        if np.issubdtype(array.dtype, np.bool_) or not np.issubdtype(array.dtype, np.integer):
            raise ValueError(f"{label} must contain integers")
        return np.asarray(array, dtype=np.int64)

    # -- observations ------------------------------------------------------------------

    def record_er_observations(self, vertex_indices, radial_layers, weights, steps: int, *, synchronize_every: int = 128):
        """Advance while recording weighted ``Er`` samples (solver.py:1080-1136).

        Samples accumulate in float64 on the device; the returned array is
        float64 with the initial state in row 0.
        """

        vertices = self._validated_index_array(vertex_indices, "vertex_indices")
        layers = self._validated_index_array(radial_layers, "radial_layers")
        w = np.asarray(weights, dtype=np.float64)
        steps = self._validated_count(steps, "step count", minimum=0)
        self._validated_count(synchronize_every, "synchronize_every", minimum=1)
        self._check_er_observation(vertices, layers, w)
        torch = self.backend.torch
        traces = torch.zeros((steps + 1, vertices.shape[0]), dtype=torch.float64, device=self.backend.torch_device)
        probe = self._engine.probe("er", vertices, np.broadcast_to(layers[:, None], vertices.shape), w)
        try:
            state = self._state()
            self._engine.sample(state, probe, traces[0])
            if steps:
                self._engine.step_sampled(state, self._source_currents(steps), steps, probe, traces[1:])
            self.steps += steps
            self.time_s = self.steps * self.time_step_s
            self.backend.synchronize()
        finally:
            probe.close()
        return self.to_numpy(traces)

    def _check_er_observation(self, vertices, layers, w) -> None:
        """Shape, range and weight checks of an Er observation set (vertices
        (R, K), layers (R,), weights (R, K)) with the reference's messages
        (solver.py:1104-1115)."""

        if vertices.ndim != 2 or w.shape != vertices.shape:
            raise ValueError("vertex_indices and weights must have matching 2-D shapes")
        if layers.shape != (vertices.shape[0],):
            raise ValueError("radial_layers must contain one layer per observation")
        if np.any(vertices < 0) or np.any(vertices >= self.mesh.n_vertices):
            raise ValueError("observation vertex index is out of range")
        if np.any(layers < 0) or np.any(layers >= len(self.radii_m)):
            raise ValueError("observation radial layer is out of range")
        if not np.all(np.isfinite(w)):
            raise ValueError("observation weights must be finite")
        if not np.allclose(w.sum(axis=1), 1.0):
            raise ValueError("observation weights must sum to one")

    def record_h_observations(
        self,
        face_indices,
        face_radial_layers,
        face_weights,
        edge_indices,
        edge_radial_layers,
        edge_weights,
        steps: int,
        *,
        synchronize_every: int = 128,
        sample_every: int = 1,
    ):
        """Advance while recording weighted ``Hr``/``Ht`` samples at H time levels
        (solver.py:1138-1229); row k holds H at (k - 1/2) dt of its sample step."""

        faces = self._validated_index_array(face_indices, "face_indices")
        face_layers = self._validated_index_array(face_radial_layers, "face_radial_layers")
        fw = np.asarray(face_weights, dtype=np.float64)
        edges = self._validated_index_array(edge_indices, "edge_indices")
        edge_layers = self._validated_index_array(edge_radial_layers, "edge_radial_layers")
        ew = np.asarray(edge_weights, dtype=np.float64)
        steps = self._validated_count(steps, "step count", minimum=0)
        synchronize_every = self._validated_count(synchronize_every, "synchronize_every", minimum=1)
        sample_every = self._validated_count(sample_every, "sample_every", minimum=1)
        if faces.ndim != 2 or fw.shape != faces.shape:
            raise ValueError("face indices and weights must have matching 2-D shapes")
        if edges.ndim != 2 or ew.shape != edges.shape:
            raise ValueError("edge indices and weights must have matching 2-D shapes")
        if face_layers.shape != faces.shape:
            raise ValueError("face radial layers must match the face indices")
        if edge_layers.shape != edges.shape:
            raise ValueError("edge radial layers must match the edge indices")
        if np.any(faces < 0) or np.any(faces >= self.mesh.n_faces):
            raise ValueError("observation face index is out of range")
        if np.any(edges < 0) or np.any(edges >= self.mesh.n_edges):
            raise ValueError("observation edge index is out of range")
        if np.any(face_layers < 0) or np.any(face_layers >= self.hr.shape[1]):
            raise ValueError("radial H observation layer is out of range")
        if np.any(edge_layers < 0) or np.any(edge_layers >= self.ht.shape[1]):
            raise ValueError("tangential H observation layer is out of range")
        if not np.all(np.isfinite(fw)) or not np.all(np.isfinite(ew)):
            raise ValueError("observation weights must be finite")
        rows = np.unique(np.concatenate((np.arange(0, steps + 1, sample_every, dtype=np.int64), np.asarray((steps,), dtype=np.int64))))
        torch = self.backend.torch
        hr_t = torch.zeros((len(rows), faces.shape[0]), dtype=torch.float64, device=self.backend.torch_device)
        ht_t = torch.zeros((len(rows), edges.shape[0]), dtype=torch.float64, device=self.backend.torch_device)
        p_hr = self._engine.probe("hr", faces, face_layers, fw)
        p_ht = self._engine.probe("ht", edges, edge_layers, ew)
        try:
            start = self.steps
            for row, target in enumerate(rows):
                if row:
                    self.step(int(target) - (self.steps - start))
                state = self._state()
                self._engine.sample(state, p_hr, hr_t[row])
                self._engine.sample(state, p_ht, ht_t[row])
                if int(target) % synchronize_every == 0:
                    self.backend.synchronize()
            self.backend.synchronize()
        finally:
            p_hr.close()
            p_ht.close()
        return self.to_numpy(hr_t), self.to_numpy(ht_t)

    # -- memory accounting -------------------------------------------------------------

    @property
    def memory_bytes(self) -> int:
        return sum(self.backend.nbytes(f) for f in (self.er, self.et, self.hr, self.ht))

    @property
    def persistent_backend_bytes(self) -> int:
        """Fields, coefficients, metric arrays, ADE state and the plan's device tables."""

        names = (
            "er", "et", "hr", "ht", "_ca_er", "_cb_er", "_ca_et", "_cb_et",
            "_primal_edge_angles", "_inverse_primal_edge_angles", "_dual_edge_angles", "_inverse_dual_edge_angles",
            "_inverse_dual_cell_solid_angles", "_inverse_face_solid_angles", "_radii", "_inverse_radii",
            "_radial_midpoints", "_inverse_radial_midpoints", "_radial_steps", "_radial_node_control_lengths",
            "_radial_center_distances",
        )
        unique = {id(getattr(self, n)): getattr(self, n) for n in names[4:]}
        total = sum(self.backend.nbytes(a) for a in unique.values())
        total += sum(self.backend.nbytes(a) for a in self._buffers.values())
        total += self._engine.plan_bytes
        if self._surface_impedance_ade is not None:
            total += self._surface_impedance_ade.persistent_bytes
        if self._plasma_coupler is not None:
            total += sum(self.backend.nbytes(j) for j in self._plasma_coupler.ade.buffers)
        return total
