"""NumPy restatement of the reference geodesic FDTD step (test oracle only).

Every function cites the reference file:line it restates (paths are relative
to the reference project root, ``src/ionosphere_fdtd/...``).  The arithmetic
follows the reference NumPy backend operation by operation so that, in
float64, this oracle reproduces the reference's own outputs to rounding
(pinned by the golden fixtures under ``tests/golden``).

Test infrastructure: imported only by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU legs.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np

# constants.py:3-6
EPSILON_0 = 8.854_187_812_8e-12
MU_0 = 1.256_637_062_12e-6
C_0 = 1.0 / (EPSILON_0 * MU_0) ** 0.5
EARTH_RADIUS_M = 6_371_000.0


# --------------------------------------------------------------------------
# Mesh (mesh.py:191-227, 386-468, 471-789)
# --------------------------------------------------------------------------


def _unit(values: np.ndarray) -> np.ndarray:
    """Row-normalise (mesh.py:471-472)."""

    return values / np.linalg.norm(values, axis=-1, keepdims=True)


def _base_icosahedron() -> tuple[np.ndarray, np.ndarray]:
    """The 12-vertex / 20-face seed (mesh.py:475-519).

    The vertex order and the face list are the reference's table: every
    index of every refined level descends from them.
    """

    g = (1.0 + np.sqrt(5.0)) / 2.0
    corners = np.array(
        [
            (-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0),
            (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
            (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1),
        ],
        dtype=np.float64,
    )
    triangles = np.array(
        [
            (0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
            (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
            (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
            (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1),
        ],
        dtype=np.int64,
    )
    return _unit(corners), _outward(_unit(corners), triangles)


def _outward(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Swap corners 1/2 of inward-facing triangles (mesh.py:558-566)."""

    out = faces.copy()
    a = vertices[out[:, 0]]
    b = vertices[out[:, 1]]
    c = vertices[out[:, 2]]
    flip = np.einsum("ij,ij->i", np.cross(b - a, c - a), a + b + c) < 0.0
    second = out[flip, 1].copy()
    out[flip, 1] = out[flip, 2]
    out[flip, 2] = second
    return out


def _rotate_to_poles(vertices: np.ndarray) -> np.ndarray:
    """Put seed vertex 5 at +z and seed vertex 9 at longitude 0 (mesh.py:522-555)."""

    src = vertices[5]
    dst = np.asarray((0.0, 0.0, 1.0))
    axis = np.cross(src, dst)
    s = np.linalg.norm(axis)
    c = float(src @ dst)
    k = np.asarray(
        (
            (0.0, -axis[2], axis[1]),
            (axis[2], 0.0, -axis[0]),
            (-axis[1], axis[0], 0.0),
        )
    )
    rot = np.eye(3) + k + k @ k * ((1.0 - c) / s**2)
    turned = vertices @ rot.T
    lon9 = np.arctan2(turned[9, 1], turned[9, 0])
    ct = np.cos(-lon9)
    st = np.sin(-lon9)
    twist = np.asarray(((ct, -st, 0.0), (st, ct, 0.0), (0.0, 0.0, 1.0)))
    return turned @ twist.T


def _quarter(vertices: np.ndarray, faces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One 4:1 refinement with midpoints numbered on first use (mesh.py:569-593)."""

    points = [row.copy() for row in vertices]
    seen: dict[tuple[int, int], int] = {}

    def mid(p: int, q: int) -> int:
        key = (p, q) if p < q else (q, p)
        index = seen.get(key)
        if index is None:
            index = len(points)
            seen[key] = index
            points.append(_unit((vertices[p] + vertices[q])[None, :])[0])
        return index

    children: list[tuple[int, int, int]] = []
    for a, b, c in faces.tolist():
        ab = mid(a, b)
        bc = mid(b, c)
        ca = mid(c, a)
        children += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
    return np.asarray(points), np.asarray(children, dtype=np.int64)


def _edge_tables(faces: np.ndarray):
    """Edges numbered in face-scan order with left/right faces (mesh.py:674-708)."""

    lookup: dict[tuple[int, int], int] = {}
    sides: list[list[tuple[int, int]]] = []
    face_edges = np.empty((len(faces), 3), dtype=np.int64)
    face_signs = np.empty_like(face_edges)
    for f, (a, b, c) in enumerate(faces.tolist()):
        for slot, (t, h) in enumerate(((a, b), (b, c), (c, a))):
            key = (t, h) if t < h else (h, t)
            sign = 1 if t < h else -1
            e = lookup.setdefault(key, len(lookup))
            if e == len(sides):
                sides.append([])
            sides[e].append((f, sign))
            face_edges[f, slot] = e
            face_signs[f, slot] = sign
    for adj in sides:
        if len(adj) != 2 or {s for _, s in adj} != {-1, 1}:
            raise RuntimeError("mesh is not a closed two-manifold")
    edges = np.asarray(list(lookup), dtype=np.int64)
    left = np.empty(len(edges), dtype=np.int64)
    right = np.empty_like(left)
    for e, adj in enumerate(sides):
        for f, s in adj:
            if s == 1:
                left[e] = f
            else:
                right[e] = f
    return edges, face_edges, face_signs, left, right


def _arc(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Great-circle angle (mesh.py:745-748)."""

    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.einsum("ij,ij->i", a, b))


def _signed_triangle(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Signed spherical triangle area (mesh.py:755-765)."""

    num = np.einsum("ij,ij->i", a, np.cross(b, c))
    den = (
        1.0
        + np.einsum("ij,ij->i", a, b)
        + np.einsum("ij,ij->i", b, c)
        + np.einsum("ij,ij->i", c, a)
    )
    return 2.0 * np.arctan2(num, den)


def _circumcentres(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Outward unit circumcentres (mesh.py:666-671)."""

    a = vertices[faces[:, 0]]
    b = vertices[faces[:, 1]]
    c = vertices[faces[:, 2]]
    n = _unit(np.cross(b - a, c - a))
    back = np.einsum("ij,ij->i", n, a + b + c) < 0.0
    n[back] *= -1.0
    return n


@dataclass
class OracleMesh:
    """Unit-sphere primal/dual tables with the reference's attribute names."""

    vertices: np.ndarray
    faces: np.ndarray
    edges: np.ndarray
    face_edges: np.ndarray
    face_edge_signs: np.ndarray
    edge_left_faces: np.ndarray
    edge_right_faces: np.ndarray
    face_centers: np.ndarray
    primal_edge_angles: np.ndarray
    dual_edge_angles: np.ndarray
    face_solid_angles: np.ndarray
    dual_cell_solid_angles: np.ndarray
    vertex_degree: np.ndarray
    subdivision: int | None = None

    @property
    def n_vertices(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.edges.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.faces.shape[0])

    def edge_midpoints(self) -> np.ndarray:
        """mesh.py:89-91."""

        return _unit(self.vertices[self.edges].sum(axis=1))


def assemble_mesh(vertices: np.ndarray, faces: np.ndarray, subdivision: int | None) -> OracleMesh:
    """Orient faces and derive every table (mesh.py:397-468, 768-789)."""

    faces = _outward(vertices, faces)
    centres = _circumcentres(vertices, faces)
    edges, face_edges, face_signs, left, right = _edge_tables(faces)
    primal = _arc(vertices[edges[:, 0]], vertices[edges[:, 1]])
    dual = _arc(centres[left], centres[right])
    face_area = np.abs(
        _signed_triangle(vertices[faces[:, 0]], vertices[faces[:, 1]], vertices[faces[:, 2]])
    )
    dual_area = np.zeros(len(vertices), dtype=np.float64)
    for end in range(2):
        owners = edges[:, end]
        wedge = _signed_triangle(vertices[owners], centres[left], centres[right])
        if end == 0:
            wedge = -wedge
        np.add.at(dual_area, owners, wedge)
    degree = np.bincount(edges.ravel(), minlength=len(vertices))
    return OracleMesh(
        vertices=vertices,
        faces=faces,
        edges=edges,
        face_edges=face_edges,
        face_edge_signs=face_signs,
        edge_left_faces=left,
        edge_right_faces=right,
        face_centers=centres,
        primal_edge_angles=primal,
        dual_edge_angles=dual,
        face_solid_angles=face_area,
        dual_cell_solid_angles=dual_area,
        vertex_degree=degree,
        subdivision=subdivision,
    )


def build_mesh(subdivision: int, orientation: str = "polar") -> OracleMesh:
    """Recursive icosahedral mesh (mesh.py:191-227, 386-394)."""

    vertices, faces = _base_icosahedron()
    if orientation == "polar":
        vertices = _rotate_to_poles(vertices)
    elif orientation != "native":
        raise ValueError("orientation must be 'native' or 'polar'")
    for _ in range(subdivision):
        vertices, faces = _quarter(vertices, faces)
    return assemble_mesh(vertices, faces, subdivision)


def vertex_incidence(mesh: Any, dtype=np.float64) -> tuple[np.ndarray, np.ndarray]:
    """Padded dual-cell incidence: tail uses first, then head uses, each in edge
    order; pad slots hold edge 0 with sign 0 (backends/numpy_backend.py:46-76)."""

    n_e = len(mesh.edges)
    owners = np.concatenate((mesh.edges[:, 0], mesh.edges[:, 1]))
    uses = np.concatenate((np.arange(n_e), np.arange(n_e)))
    signs = np.concatenate((np.ones(n_e), -np.ones(n_e))).astype(dtype)
    order = np.argsort(owners, kind="stable")
    owners, uses, signs = owners[order], uses[order], signs[order]
    counts = np.bincount(owners, minlength=len(mesh.vertices))
    starts = np.cumsum(np.concatenate(([0], counts[:-1])))
    slot = np.arange(len(owners)) - np.repeat(starts, counts)
    width = int(counts.max())
    table = np.zeros((len(mesh.vertices), width), dtype=np.int64)
    table_signs = np.zeros((len(mesh.vertices), width), dtype=dtype)
    table[owners, slot] = uses
    table_signs[owners, slot] = signs
    return table, table_signs


# --------------------------------------------------------------------------
# Materials, sources, surface impedance, plasma (setup restatements)
# --------------------------------------------------------------------------


@dataclass
class EarthIonosphereParams:
    """Parameters of materials.py:242-281 (anomalies omitted)."""

    lithosphere_conductivity_s_m: float = 1.0e-3
    lithosphere_relative_permittivity: float = 10.0
    atmosphere_relative_permittivity: float = 1.0
    ionosphere_reference_height_m: float = 74_000.0
    ionosphere_scale_height_m: float = 6_000.0
    ionosphere_prefactor_hz: float = 2.5e5

    def sample(self, directions, altitudes_m, earth_radius_m):
        return earth_ionosphere_sample(self, directions, altitudes_m)


def earth_ionosphere_sample(p: EarthIonosphereParams, directions, altitudes_m):
    """Exponential ionosphere over a homogeneous lithosphere (materials.py:283-326)."""

    h = np.asarray(altitudes_m, dtype=np.float64)
    air = (
        p.ionosphere_prefactor_hz
        * EPSILON_0
        * np.exp(np.clip((h - p.ionosphere_reference_height_m) / p.ionosphere_scale_height_m, -80.0, 80.0))
    )
    ground = h < 0.0
    sigma = np.where(ground, p.lithosphere_conductivity_s_m, air)
    eps = np.where(ground, p.lithosphere_relative_permittivity, p.atmosphere_relative_permittivity)
    n = len(directions)
    return (
        np.broadcast_to(sigma, (n, len(h))).copy(),
        np.broadcast_to(eps, (n, len(h))).copy(),
    )


def geographic_direction(lat: float, lon: float) -> np.ndarray:
    """sources.py:18-32."""

    a = np.deg2rad(lat)
    o = np.deg2rad(lon)
    return np.asarray((np.cos(a) * np.cos(o), np.cos(a) * np.sin(o), np.sin(a)), dtype=np.float64)


def geographic_face_index(mesh: Any, lat: float, lon: float) -> int:
    """Face containing a direction, nearest circumcentre on ties (sources.py:53-85)."""

    d = geographic_direction(lat, lon)
    tri = mesh.vertices[mesh.faces]
    sides = np.column_stack(
        [np.einsum("ij,j->i", np.cross(tri[:, k], tri[:, (k + 1) % 3]), d) for k in range(3)]
    )
    inside = np.all(sides >= -1.0e-12, axis=1) | np.all(sides <= 1.0e-12, axis=1)
    cand = np.flatnonzero(inside)
    if len(cand):
        return int(cand[np.argmax(mesh.face_centers[cand] @ d)])
    return int(np.argmax(mesh.face_centers @ d))


def geographic_distribution(mesh: Any, altitudes_m, lat: float, lon: float, alt: float):
    """Barycentric weights of the containing triangle (sources.py:88-124)."""

    d = geographic_direction(lat, lon)
    f = geographic_face_index(mesh, lat, lon)
    corners = mesh.faces[f]
    pa, pb, pc = mesh.vertices[corners]
    normal = np.cross(pb - pa, pc - pa)
    hit = d * float((normal @ pa) / (normal @ d))
    ab = pb - pa
    ac = pc - pa
    off = hit - pa
    aa, bc_, cc = float(ab @ ab), float(ab @ ac), float(ac @ ac)
    oa, oc = float(off @ ab), float(off @ ac)
    den = aa * cc - bc_**2
    wb = (cc * oa - bc_ * oc) / den
    wc = (aa * oc - bc_ * oa) / den
    w = np.clip(np.asarray((1.0 - wb - wc, wb, wc)), 0.0, None)
    w /= w.sum()
    layer = int(np.argmin(np.abs(np.asarray(altitudes_m) - alt)))
    return corners.copy(), layer, w


def radial_linear_distribution(levels, alt: float):
    """Exact two-plane split of an altitude (sources.py:127-154)."""

    levels = np.asarray(levels, dtype=np.float64)
    if alt < levels[0] or alt > levels[-1]:
        raise ValueError("source altitude is outside the radial grid")
    up = int(np.searchsorted(levels, alt, side="left"))
    if up < len(levels) and levels[up] == alt:
        return np.asarray((up,), dtype=np.int64), np.asarray((1.0,))
    lo = up - 1
    wu = (alt - levels[lo]) / (levels[up] - levels[lo])
    return np.asarray((lo, up), dtype=np.int64), np.asarray((1.0 - wu, wu))


@dataclass
class OracleSource:
    """Gaussian current (sources.py:157-254) and its tangential form (257-335)."""

    latitude_deg: float = 35.1595
    longitude_deg: float = 126.8526
    altitude_m: float = 2_500.0
    peak_current_a: float = 1.0e6
    vertical_element_length_m: float = 5_000.0
    center_time_s: float | None = None
    one_over_e_half_width_s: float | None = None
    carrier_frequency_hz: float = 0.0
    tangential: bool = False
    azimuths_deg: tuple[float, ...] = (0.0,)
    line_lengths_m: tuple[float, ...] | None = None
    edge_assignment: str = "projected"

    def current_a(self, t: float, dt: float) -> float:
        """sources.py:237-254."""

        if self.one_over_e_half_width_s is not None:
            w = self.one_over_e_half_width_s
        elif self.carrier_frequency_hz:
            w = 0.5 / self.carrier_frequency_hz
        else:
            w = 12.0 * dt
        t0 = self.center_time_s if self.center_time_s is not None else max(4.0 * w, 36.0 * dt)
        env = np.exp(-(((t - t0) / w) ** 2))
        if self.carrier_frequency_hz:
            env *= np.cos(2.0 * np.pi * self.carrier_frequency_hz * (t - t0))
        return float(self.peak_current_a * env)


def staggered_distribution(src: OracleSource, mesh, altitudes_m):
    """Vertical source supports (sources.py:220-235)."""

    corners, _, hw = geographic_distribution(mesh, altitudes_m, src.latitude_deg, src.longitude_deg, src.altitude_m)
    layers, rw = radial_linear_distribution(altitudes_m, src.altitude_m)
    n = len(layers)
    return np.repeat(corners, n), np.tile(layers, len(corners)), np.repeat(hw, n) * np.tile(rw, len(corners))


def tangential_distribution(src: OracleSource, mesh, earth_radius_m, midpoint_altitudes_m):
    """Ground-line currents projected on the containing face's edges (sources.py:290-335)."""

    f = geographic_face_index(mesh, src.latitude_deg, src.longitude_deg)
    fe = mesh.face_edges[f].copy()
    ends = mesh.vertices[mesh.edges[fe]]
    dirs = ends[:, 1] - ends[:, 0]
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    lat = np.deg2rad(src.latitude_deg)
    lon = np.deg2rad(src.longitude_deg)
    east = np.asarray((-np.sin(lon), np.cos(lon), 0.0))
    north = np.asarray((-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)))
    lengths = mesh.primal_edge_angles[fe] * (earth_radius_m + src.altitude_m)
    w = np.zeros(len(fe))
    lines = src.line_lengths_m or tuple(1.0 for _ in src.azimuths_deg)
    for az, ll in zip(src.azimuths_deg, lines):
        a = np.deg2rad(az)
        want = np.cos(a) * north + np.sin(a) * east
        proj = dirs @ want
        if src.edge_assignment == "projected":
            w += ll * proj / lengths
        else:
            k = int(np.argmax(np.abs(proj)))
            w[k] += ll * proj[k] / lengths[k]
    layers, rw = radial_linear_distribution(midpoint_altitudes_m, src.altitude_m)
    return np.repeat(fe, len(layers)), np.tile(layers, len(fe)), np.repeat(w, len(layers)) * np.tile(rw, len(fe))


@dataclass
class OracleSurface:
    """Diffusive conductive half-space (surface_impedance.py:14-111)."""

    conductivity_s_m: Any
    minimum_frequency_hz: float = 5.0
    maximum_frequency_hz: float = 45.0
    terms: int = 16
    pole_span_decades: float = 5.0
    permeability_h_m: float = MU_0

    def poles(self) -> np.ndarray:
        """surface_impedance.py:66-75."""

        lo = np.log(2.0 * np.pi * self.minimum_frequency_hz) - self.pole_span_decades * np.log(10.0)
        hi = np.log(2.0 * np.pi * self.maximum_frequency_hz) + self.pole_span_decades * np.log(10.0)
        step = (hi - lo) / self.terms
        return np.exp(lo + (np.arange(self.terms) + 0.5) * step)

    def weights(self) -> np.ndarray:
        """surface_impedance.py:77-90."""

        p = self.poles()
        if self.terms > 1:
            spacing = np.log(p[-1] / p[0]) / (self.terms - 1)
        else:
            spacing = np.log(self.maximum_frequency_hz / self.minimum_frequency_hz) + 2.0 * self.pole_span_decades * np.log(10.0)
        return spacing * np.sqrt(p) / np.pi

    def per_edge(self, n_edges: int) -> np.ndarray:
        """surface_impedance.py:92-111."""

        s = np.asarray(self.conductivity_s_m, dtype=np.float64).reshape(-1)
        if s.size == 1:
            return np.full(n_edges, s[0])
        if s.size != n_edges:
            raise ValueError("surface conductivity does not match mesh edges")
        return s.copy()


@dataclass
class OracleSpecies:
    """One charged fluid on faces x radial midpoints (plasma.py:32-61)."""

    charge_c: float
    mass_kg: float
    number_density_m3: np.ndarray
    collision_frequency_hz: np.ndarray


@dataclass
class OraclePlasma:
    """Magnetic field and species on faces x midpoints (plasma.py:64-113)."""

    magnetic_field_t: np.ndarray
    species: list = field(default_factory=list)


# --------------------------------------------------------------------------
# Solver (solver.py:174-1294 on the NumPy backend)
# --------------------------------------------------------------------------


class OracleFDTD:
    """NumPy restatement of ``GeodesicFDTD`` with the NumPy backend."""

    def __init__(
        self,
        *,
        subdivision: int = 2,
        radial_cells: int = 24,
        minimum_altitude_m: float = -100_000.0,
        maximum_altitude_m: float = 100_000.0,
        earth_radius_m: float = EARTH_RADIUS_M,
        courant_factor: float = 0.35,
        time_step_s: float | None = None,
        radial_altitudes_m=None,
        geometry_mode: str = "full-spherical",
        loss_integration: str = "exponential",
        compress: bool = False,
        material: Any = None,
        source: OracleSource | None = None,
        surface: OracleSurface | None = None,
        plasma: OraclePlasma | None = None,
        mesh: Any = None,
        orientation: str = "polar",
        dtype=np.float64,
    ) -> None:
        self.dtype = np.dtype(dtype)
        self.mesh = mesh if mesh is not None else build_mesh(subdivision, orientation)
        self.full = geometry_mode == "full-spherical"
        self.compress = compress
        m = self.mesh
        # radial grid: solver.py:260-283
        if radial_altitudes_m is None:
            self.altitudes_m = np.linspace(minimum_altitude_m, maximum_altitude_m, radial_cells + 1)
        else:
            self.altitudes_m = np.asarray(radial_altitudes_m, dtype=np.float64)
        self.earth_radius_m = earth_radius_m
        self.radii_m = earth_radius_m + self.altitudes_m
        self.midpoints_m = 0.5 * (self.radii_m[:-1] + self.radii_m[1:])
        self.midpoint_altitudes_m = self.midpoints_m - earth_radius_m
        self.steps_m = np.diff(self.radii_m)
        ctrl = np.empty(len(self.radii_m))
        ctrl[0] = 0.5 * self.steps_m[0]
        ctrl[-1] = 0.5 * self.steps_m[-1]
        ctrl[1:-1] = np.diff(self.midpoints_m)
        self.control_m = ctrl
        material = material if material is not None else EarthIonosphereParams()
        # point material support: solver.py:522-531, 579-581
        self.sigma_er, self.eps_er = (
            np.asarray(a, dtype=np.float64)
            for a in material.sample(m.vertices, self.altitudes_m, earth_radius_m)
        )
        self.sigma_et, self.eps_et = (
            np.asarray(a, dtype=np.float64)
            for a in material.sample(m.edge_midpoints(), self.midpoint_altitudes_m, earth_radius_m)
        )
        self.plasma = plasma
        self.cfl_limit_s = self._cfl()
        dt_max = courant_factor * self.cfl_limit_s
        self.dt = time_step_s if time_step_s is not None else dt_max
        if self.dt > dt_max * (1.0 + 1.0e-12):
            raise ValueError("time step exceeds conservative limit")
        self.source = source
        shape_n = (m.n_vertices, len(self.radii_m))
        self.er = np.zeros(shape_n, dtype=self.dtype)
        self.ht = np.zeros((m.n_edges, len(self.radii_m)), dtype=self.dtype)
        self.et = np.zeros((m.n_edges, len(self.midpoints_m)), dtype=self.dtype)
        self.hr = np.zeros((m.n_faces, len(self.midpoints_m)), dtype=self.dtype)
        self._setup_surface(surface)
        self._setup_plasma(plasma)
        self._setup_geometry()
        self._setup_coefficients(loss_integration)
        self._setup_sources()
        self.steps = 0
        self.time_s = 0.0

    # -- setup --------------------------------------------------------------

    def _a(self, values) -> np.ndarray:
        return np.array(values, dtype=self.dtype, copy=True)

    def _cfl(self) -> float:
        """solver.py:377-406."""

        r0 = float(self.radii_m.min())
        p = r0 * float(self.mesh.primal_edge_angles.min())
        d = r0 * float(self.mesh.dual_edge_angles.min())
        rr = float(self.steps_m.min())
        inv2 = p**-2 + d**-2 + (2.0 / rr) ** 2
        eps_min = min(float(np.min(self.eps_er)), float(np.min(self.eps_et)))
        limit = np.sqrt(eps_min) / (C_0 * np.sqrt(inv2))
        if self.plasma is None:
            return limit
        drive = np.zeros(self.plasma.magnetic_field_t.shape[:2])
        for sp in self.plasma.species:
            drive += sp.number_density_m3 * sp.charge_c**2 / sp.mass_kg
        wp = np.sqrt(float(np.max(drive)) / (EPSILON_0 * eps_min))
        if wp == 0.0:
            return limit
        return min(limit, 2.0 / wp)

    def _setup_geometry(self) -> None:
        """solver.py:408-442 plus backend tables (numpy_backend.py:12-76)."""

        m = self.mesh
        self.g_primal = self._a(m.primal_edge_angles[:, None])
        self.g_inv_primal = self._a(1.0 / m.primal_edge_angles[:, None])
        self.g_dual = self._a(m.dual_edge_angles[:, None])
        self.g_inv_dual = self._a(1.0 / m.dual_edge_angles[:, None])
        self.g_inv_dual_area = self._a(1.0 / m.dual_cell_solid_angles[:, None])
        self.g_inv_face_area = self._a(1.0 / m.face_solid_angles[:, None])
        self.r = self._a(self.radii_m)
        self.inv_r = self._a(1.0 / self.radii_m[None, :])
        self.mid = self._a(self.midpoints_m)
        self.inv_mid = self._a(1.0 / self.midpoints_m[None, :])
        self.dr = self._a(self.steps_m)
        self.ctrl = self._a(self.control_m)
        self.cd = self._a(self.midpoints_m[1:] - self.midpoints_m[:-1])
        self.face_signs = np.array(m.face_edge_signs, dtype=self.dtype)
        self.v_edges, self.v_signs = vertex_incidence(m, self.dtype)

    def _setup_coefficients(self, loss: str) -> None:
        """solver.py:706-761."""

        e_er = EPSILON_0 * self.eps_er
        e_et = EPSILON_0 * self.eps_et
        dt = self.dt

        def expo(sig, eps):
            rate = sig * dt / eps
            decay = np.exp(-rate)
            phi = np.ones_like(rate)
            nz = rate != 0.0
            phi[nz] = -np.expm1(-rate[nz]) / rate[nz]
            return decay, dt / eps * phi

        def trap(sig, eps):
            q = sig * dt / (2.0 * eps)
            return (1.0 - q) / (1.0 + q), dt / (eps * (1.0 + q))

        rule = trap if loss == "trapezoidal" else expo
        ca_er, cb_er = rule(self.sigma_er, e_er)
        ca_et, cb_et = rule(self.sigma_et, e_et)
        if self.compress:
            ca_er, cb_er, ca_et, cb_et = (v[:1] for v in (ca_er, cb_er, ca_et, cb_et))
        self.ca_er, self.cb_er = self._a(ca_er), self._a(cb_er)
        self.ca_et, self.cb_et = self._a(ca_et), self._a(cb_et)

    def _setup_sources(self) -> None:
        """solver.py:347-362."""

        self.src_v = self.src_t = None
        if self.source is None:
            return
        if self.source.tangential:
            e, k, w = tangential_distribution(self.source, self.mesh, self.earth_radius_m, self.midpoint_altitudes_m)
            self.src_t = (e.astype(np.int64), k.astype(np.int64), self._a(w))
        else:
            v, k, w = staggered_distribution(self.source, self.mesh, self.altitudes_m)
            self.src_v = (v.astype(np.int64), k.astype(np.int64), self._a(w))

    def _setup_surface(self, surface: OracleSurface | None) -> None:
        """surface_impedance.py:176-203."""

        self.surface = surface
        if surface is None:
            return
        p = surface.poles()
        w = surface.weights()
        a = 0.5 * self.dt * p
        self.si_decay = self._a((1.0 - a) / (1.0 + a))
        self.si_drive = self._a(a / (1.0 + a))
        self.si_hist = self._a(w / (1.0 + a))
        self.si_scale = self._a(np.sqrt(surface.permeability_h_m / surface.per_edge(self.mesh.n_edges)))
        self.si_memory = np.zeros((self.mesh.n_edges, surface.terms), dtype=self.dtype)

    def _setup_plasma(self, plasma: OraclePlasma | None) -> None:
        """plasma.py:374-411, 458-487, 548-588."""

        if plasma is None:
            return
        m = self.mesh
        dt = self.dt
        # face reconstruction (plasma.py:548-559)
        nrm = np.cross(m.vertices[m.edges[:, 0]], m.vertices[m.edges[:, 1]])
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        tang = np.cross(nrm[m.face_edges], m.face_centers[:, None, :])
        tang /= np.linalg.norm(tang, axis=2, keepdims=True)
        recon = np.empty_like(tang)
        for f in range(m.n_faces):
            recon[f] = np.linalg.pinv(tang[f]).T
        # edge slots within left/right faces (plasma.py:562-569)
        idx = np.arange(m.n_edges)[:, None]
        lslot = np.argmax(m.face_edges[m.edge_left_faces] == idx, axis=1)
        rslot = np.argmax(m.face_edges[m.edge_right_faces] == idx, axis=1)
        # vertex area-weighted face average (plasma.py:572-588)
        inc: list[list[int]] = [[] for _ in range(m.n_vertices)]
        for f, tri in enumerate(m.faces.tolist()):
            for v in tri:
                inc[v].append(f)
        width = max(len(x) for x in inc)
        vf = np.zeros((m.n_vertices, width), dtype=np.int64)
        vw = np.zeros((m.n_vertices, width))
        for v, fl in enumerate(inc):
            fi = np.asarray(fl, dtype=np.int64)
            ww = m.face_solid_angles[fi]
            ww /= np.sum(ww)
            vf[v, : len(fl)] = fi
            vw[v, : len(fl)] = ww
        self.p_recon = self._a(recon)
        self.p_centres = self._a(m.face_centers)
        self.p_ltan = self._a(tang[m.edge_left_faces, lslot])
        self.p_rtan = self._a(tang[m.edge_right_faces, rslot])
        self.p_vfaces = vf
        self.p_vweights = self._a(vw)
        # ADE coefficients (plasma.py:374-411)
        bmag = np.linalg.norm(plasma.magnetic_field_t, axis=2)
        bdir = np.zeros_like(plasma.magnetic_field_t)
        nz = bmag > 0.0
        bdir[nz] = plasma.magnetic_field_t[nz] / bmag[nz, None]
        self.p_b = self._a(bdir)
        self.p_coef = []
        self.p_current = []
        for sp in plasma.species:
            nu = sp.collision_frequency_hz
            gyro = sp.charge_c * bmag / sp.mass_kg
            decay = np.exp(-nu * dt)
            angle = gyro * dt
            eig = -nu + 1j * gyro
            integ = np.expm1(eig * dt) / eig
            par = -np.expm1(-nu * dt) / nu
            drive = sp.number_density_m3 * sp.charge_c**2 / sp.mass_kg
            self.p_coef.append(
                tuple(self._a(v) for v in (decay, np.cos(angle), np.sin(angle), drive * par, drive * integ.real, drive * integ.imag))
            )
            self.p_current.append(np.zeros((*bmag.shape, 3), dtype=self.dtype))

    # -- primitives (numpy_backend.py:93-114) --------------------------------

    def _edge_difference(self, values):
        return values[self.mesh.edges[:, 1]] - values[self.mesh.edges[:, 0]]

    def _dual_edge_difference(self, values):
        return values[self.mesh.edge_left_faces] - values[self.mesh.edge_right_faces]

    def _face_circulation(self, values):
        picked = values[self.mesh.face_edges]
        s = self.face_signs
        while s.ndim < picked.ndim:
            s = s[..., None]
        return np.sum(picked * s, axis=1)

    def _dual_cell_circulation(self, values):
        shape = (self.mesh.n_vertices,) + (1,) * (values.ndim - 1)
        out = values[self.v_edges[:, 0]].copy()
        out *= self.v_signs[:, 0].reshape(shape)
        for k in range(1, self.v_edges.shape[1]):
            out += values[self.v_edges[:, k]] * self.v_signs[:, k].reshape(shape)
        return out

    # -- radial stencils (solver.py:443-465) ---------------------------------

    def _d_et(self):
        vals = self.et
        if self.full:
            vals = vals * self.mid[None, :]
        out = np.empty_like(self.ht)
        out[:, 0] = 2.0 * vals[:, 0] / self.dr[0]
        out[:, -1] = -2.0 * vals[:, -1] / self.dr[-1]
        if self.ht.shape[1] > 2:
            out[:, 1:-1] = np.diff(vals, axis=1) / self.cd
        if self.full:
            out *= self.inv_r
        return out

    def _d_ht(self):
        vals = self.ht
        if self.full:
            vals = vals * self.r[None, :]
        out = np.diff(vals, axis=1) / self.dr[None, :]
        if self.full:
            out *= self.inv_mid
        return out

    # -- ADEs ----------------------------------------------------------------

    def _surface_advance(self, h_old, e1, g0):
        """surface_impedance.py:225-270."""

        hist = self.si_scale * (self.si_memory * self.si_hist[None, :]).sum(axis=1)
        gain = self.si_scale * self.si_hist.sum()
        k = 2.0 * self.dt / (MU_0 * self.dr[0])
        force = self.dt / MU_0 * g0
        c = k * gain
        h_new = ((1.0 - 0.5 * c) * h_old + force - k * e1 + k * hist) / (1.0 + 0.5 * c)
        self.si_memory[:] = self.si_memory * self.si_decay[None, :] + (h_new + h_old)[:, None] * self.si_drive[None, :]
        return h_new

    @staticmethod
    def _cross(v, b):
        """plasma.py:591-596."""

        out = np.empty_like(v)
        out[..., 0] = v[..., 1] * b[..., 2] - v[..., 2] * b[..., 1]
        out[..., 1] = v[..., 2] * b[..., 0] - v[..., 0] * b[..., 2]
        out[..., 2] = v[..., 0] * b[..., 1] - v[..., 1] * b[..., 0]
        return out

    def _plasma_advance(self):
        """Face-vector E, per-species current update, scatter to Er/Et supports
        (plasma.py:413-442, 489-527)."""

        m = self.mesh
        nodes = self.er[m.faces].sum(axis=1) / 3.0
        radial = 0.5 * (nodes[:, :-1] + nodes[:, 1:])
        ev = self.et[m.face_edges]
        tang = (ev[..., None] * self.p_recon[:, :, None, :]).sum(axis=1)
        efield = tang + radial[..., None] * self.p_centres[:, None, :]
        b = self.p_b
        total = np.zeros(efield.shape, dtype=self.dtype)
        e_par = (efield * b).sum(axis=2)[..., None] * b
        e_perp = efield - e_par
        e_x = self._cross(e_perp, b)
        for i, (decay, cs, sn, dpar, dre, dim) in enumerate(self.p_coef):
            j = self.p_current[i]
            j_par = (j * b).sum(axis=2)[..., None] * b
            j_perp = j - j_par
            j_x = self._cross(j_perp, b)
            new = (
                decay[..., None] * j_par
                + dpar[..., None] * e_par
                + decay[..., None] * (cs[..., None] * j_perp + sn[..., None] * j_x)
                + dre[..., None] * e_perp
                + dim[..., None] * e_x
            )
            self.p_current[i][:] = new
            total += new
        left = (total[m.edge_left_faces] * self.p_ltan[:, None, :]).sum(axis=2)
        right = (total[m.edge_right_faces] * self.p_rtan[:, None, :]).sum(axis=2)
        jt = 0.5 * (left + right)
        at_faces = (total * self.p_centres[:, None, :]).sum(axis=2)
        at_vertices = (at_faces[self.p_vfaces] * self.p_vweights[:, :, None]).sum(axis=1)
        jr = np.zeros((at_vertices.shape[0], at_vertices.shape[1] + 1), dtype=self.dtype)
        jr[:, 0] = at_vertices[:, 0]
        jr[:, -1] = at_vertices[:, -1]
        if at_vertices.shape[1] > 1:
            jr[:, 1:-1] = 0.5 * (at_vertices[:, :-1] + at_vertices[:, 1:])
        return jr, jt

    # -- the step (solver.py:867-989) ----------------------------------------

    def update_magnetic(self) -> None:
        """solver.py:877-921."""

        g = self._edge_difference(self.er)
        g *= self.g_inv_primal
        g *= self.inv_r
        if self.surface is not None:
            g0 = g[:, 0] + 0.0
            h_old = self.ht[:, 0] + 0.0
        d = self._d_et()
        g -= d
        g *= self.dt / MU_0
        self.ht += g
        if self.surface is not None:
            metric = self.midpoints_m[0] / self.radii_m[0] if self.full else 1.0
            self.ht[:, 0] = self._surface_advance(h_old, metric * self.et[:, 0], g0)
        circ = self._face_circulation(self.et * self.g_primal)
        circ *= self.g_inv_face_area
        circ *= self.inv_mid
        circ *= self.dt / MU_0
        self.hr -= circ

    def update_electric(self, current_a: float = 0.0) -> None:
        """solver.py:923-989."""

        pc = self._plasma_advance() if self.plasma is not None else None
        mc = self._dual_cell_circulation(self.ht * self.g_dual)
        mc *= self.g_inv_dual_area
        mc *= self.inv_r
        dens = None
        if self.src_v is not None:
            v, k, w = self.src_v
            dens = w * current_a * self.source.vertical_element_length_m * self.g_inv_dual_area[v, 0] / self.r[k] ** 2 / self.ctrl[k]
        self.er *= self.ca_er
        mc *= self.cb_er
        self.er += mc
        if dens is not None:
            v, k, _ = self.src_v
            cv = 0 if self.compress else v
            self.er[v, k] -= self.cb_er[cv, k] * dens
        if pc is not None:
            self.er -= self.cb_er * pc[0]
        g = self._dual_edge_difference(self.hr)
        g *= self.g_inv_dual
        g *= self.inv_mid
        g -= self._d_ht()
        self.et *= self.ca_et
        g *= self.cb_et
        self.et += g
        if self.src_t is not None:
            e, k, w = self.src_t
            dens_t = w * current_a * self.g_inv_dual[e, 0] / self.mid[k] / self.dr[k]
            ce = 0 if self.compress else e
            self.et[e, k] -= self.cb_et[ce, k] * dens_t
        if pc is not None:
            self.et -= self.cb_et * pc[1]

    def current_at(self, step_index: int) -> float:
        """Waveform sampled at the half step (solver.py:805-813, 851-865)."""

        if self.source is None:
            return 0.0
        return self.source.current_a((step_index + 0.5) * self.dt, self.dt)

    def step(self, count: int = 1) -> None:
        """solver.py:789-816 (eager path)."""

        for _ in range(count):
            current = self.current_at(self.steps)
            self.update_magnetic()
            self.update_electric(current)
            self.steps += 1
            self.time_s = self.steps * self.dt

    def record_er(self, vertices, layers, weights, steps: int) -> np.ndarray:
        """Weighted Er samples, initial row first (solver.py:1080-1136)."""

        vertices = np.asarray(vertices, dtype=np.int64)
        layers = np.asarray(layers, dtype=np.int64)
        w = self._a(weights)
        traces = np.zeros((steps + 1, vertices.shape[0]), dtype=self.dtype)

        def sample(row):
            traces[row] = (self.er[vertices, layers[:, None]] * w).sum(axis=1)

        sample(0)
        for i in range(steps):
            self.step(1)
            sample(i + 1)
        return traces

    def record_h(self, faces, face_layers, face_weights, edges, edge_layers, edge_weights, steps: int, sample_every: int = 1):
        """Weighted Hr/Ht samples at H time levels (solver.py:1138-1229)."""

        faces = np.asarray(faces, dtype=np.int64)
        fl = np.asarray(face_layers, dtype=np.int64)
        fw = self._a(face_weights)
        edges = np.asarray(edges, dtype=np.int64)
        el = np.asarray(edge_layers, dtype=np.int64)
        ew = self._a(edge_weights)
        rows = np.unique(np.concatenate((np.arange(0, steps + 1, sample_every), [steps])))
        hr_t = np.zeros((len(rows), faces.shape[0]), dtype=self.dtype)
        ht_t = np.zeros((len(rows), edges.shape[0]), dtype=self.dtype)

        def sample(row):
            hr_t[row] = (self.hr[faces, fl] * fw).sum(axis=1)
            ht_t[row] = (self.ht[edges, el] * ew).sum(axis=1)

        sample(0)
        done = 0
        for row, target in enumerate(rows[1:], start=1):
            self.step(int(target) - done)
            done = int(target)
            sample(row)
        return hr_t, ht_t

    def max_abs(self) -> dict[str, float]:
        """The four field maxima of diagnostics() (solver.py:1027-1030)."""

        return {name: float(np.max(np.abs(getattr(self, name)))) for name in ("er", "et", "hr", "ht")}
