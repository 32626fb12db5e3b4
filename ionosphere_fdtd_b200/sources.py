"""Gaussian current sources and their deposition on the staggered grid.

Same waveform, locations and support weights as the reference
(sources.py:18-335).  The waveform is evaluated on the host in float64 for
each step, exactly where the reference evaluates it; the CUDA step kernel
applies the precomputed support coefficients.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import TYPE_CHECKING

import numpy as np
from numpy.typing import NDArray

if TYPE_CHECKING:
    from .solver import GeodesicFDTD

GWANGJU_LATITUDE_DEG = 35.1595
GWANGJU_LONGITUDE_DEG = 126.8526


def geographic_direction(latitude_deg: float, longitude_deg: float) -> NDArray[np.float64]:
    lat = np.deg2rad(latitude_deg)
    lon = np.deg2rad(longitude_deg)
    return np.asarray((np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)), dtype=np.float64)


def geographic_tangent_basis(latitude_deg: float, longitude_deg: float):
    """Local east and north unit vectors."""

    lat = np.deg2rad(latitude_deg)
    lon = np.deg2rad(longitude_deg)
    east = np.asarray((-np.sin(lon), np.cos(lon), 0.0))
    north = np.asarray((-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)))
    return east, north


@dataclass(frozen=True)
class _FaceSearch:
    """Per-mesh search structure: the search cone and the faces sorted by the z
    coordinate of their circumcentre."""

    mesh: object
    half_angle: float  # of the search cone, radians
    cos_limit: float  # its cosine
    order: NDArray[np.int64]  # face indices by ascending circumcentre z
    z: NDArray[np.float64]  # those z values


_SEARCH_CACHE: dict[int, _FaceSearch] = {}
_BAND_MARGIN = 1.0e-6  # radians and z units added to each band; the band only needs to hold the cone


def _face_search(mesh) -> _FaceSearch:
    """The search cone holds every face: its half-angle is 1 % above the largest
    angle between a face's circumcentre and its corners, plus 1e-6 rad."""

    hit = _SEARCH_CACHE.get(id(mesh))
    if hit is not None and hit.mesh is mesh:
        return hit
    cos_min = 1.0
    for lo in range(0, mesh.n_faces, 1 << 20):
        corners = mesh.vertices[mesh.faces[lo : lo + (1 << 20)]]
        centres = mesh.face_centers[lo : lo + (1 << 20)]
        cos_min = min(cos_min, float(np.min(np.einsum("fkj,fj->fk", corners, centres))))
    half = min(np.pi, 1.01 * float(np.arccos(np.clip(cos_min, -1.0, 1.0))) + 1.0e-6)
    z = np.ascontiguousarray(mesh.face_centers[:, 2])
    order = np.argsort(z, kind="stable")
    out = _FaceSearch(mesh, half, float(np.cos(half)), order, z[order])
    if len(_SEARCH_CACHE) >= 4:
        _SEARCH_CACHE.clear()
    _SEARCH_CACHE[id(mesh)] = out
    return out


def _cone_band(search: _FaceSearch, u: NDArray[np.float64]) -> NDArray[np.int64]:
    """Faces whose circumcentre z lies in the band that any direction within the
    search cone around the unit vector ``u`` can reach (a superset of the cone)."""

    theta = float(np.arccos(np.clip(u[2], -1.0, 1.0)))
    a = search.half_angle + _BAND_MARGIN
    z_lo = float(np.cos(min(np.pi, theta + a))) - _BAND_MARGIN
    z_hi = float(np.cos(max(0.0, theta - a))) + _BAND_MARGIN
    lo = int(np.searchsorted(search.z, z_lo, side="left"))
    hi = int(np.searchsorted(search.z, z_hi, side="right"))
    return search.order[lo:hi]


def geographic_face_index(simulation, latitude_deg: float, longitude_deg: float) -> int:
    """Face containing the direction; nearest circumcentre among ties (sources.py:53-85).

    The containment test runs only on faces whose circumcentre lies within
    the search cone of the direction or of its antipode (the test also
    accepts a face that holds the antipode); every face the test can accept
    lies in that set.  The cone's faces are found in two z bands of the
    faces sorted by circumcentre z, and are tested in index order, so the
    candidates, their order and the choice (the reference's own product
    ``face_centers[candidates] @ direction``) are those of the test over all
    faces."""

    d = geographic_direction(latitude_deg, longitude_deg)
    mesh = simulation.mesh
    centres = mesh.face_centers
    search = _face_search(mesh)
    pool = np.unique(np.concatenate((_cone_band(search, d), _cone_band(search, -d))))
    proximity = centres[pool] @ d
    near = pool[(proximity >= search.cos_limit) | (-proximity >= search.cos_limit)]
    tri = mesh.vertices[mesh.faces[near]]
    sides = np.column_stack([np.einsum("ij,j->i", np.cross(tri[:, k], tri[:, (k + 1) % 3]), d) for k in range(3)])
    inside = np.all(sides >= -1.0e-12, axis=1) | np.all(sides <= 1.0e-12, axis=1)
    cand = near[inside]
    return int(cand[np.argmax(centres[cand] @ d)]) if len(cand) else int(np.argmax(centres @ d))


def geographic_distribution(simulation, latitude_deg: float, longitude_deg: float, altitude_m: float):
    """Triangle vertices, nearest radial layer and barycentric weights (sources.py:88-124)."""

    d = geographic_direction(latitude_deg, longitude_deg)
    f = geographic_face_index(simulation, latitude_deg, longitude_deg)
    corners = simulation.mesh.faces[f]
    pa, pb, pc = simulation.mesh.vertices[corners]
    normal = np.cross(pb - pa, pc - pa)
    hit = d * float((normal @ pa) / (normal @ d))
    ab, ac, off = pb - pa, pc - pa, hit - pa
    d_bb, d_bc, d_cc = float(ab @ ab), float(ab @ ac), float(ac @ ac)
    d_ob, d_oc = float(off @ ab), float(off @ ac)
    den = d_bb * d_cc - d_bc**2
    wb = (d_cc * d_ob - d_bc * d_oc) / den
    wc = (d_bb * d_oc - d_bc * d_ob) / den
    weights = np.clip(np.asarray((1.0 - wb - wc, wb, wc)), 0.0, None)
    weights /= weights.sum()
    layer = int(np.argmin(np.abs(simulation.altitudes_m - altitude_m)))
    return corners.copy(), layer, weights


def radial_linear_distribution(radial_altitudes_m, altitude_m: float):
    """Split an altitude exactly between the two bracketing planes (sources.py:127-154)."""

    levels = np.asarray(radial_altitudes_m, dtype=np.float64)
    if levels.ndim != 1 or len(levels) < 1:
        raise ValueError("radial_altitudes_m must be a nonempty 1-D array")
    if not np.all(np.diff(levels) > 0.0):
        raise ValueError("radial_altitudes_m must be strictly increasing")
    if altitude_m < levels[0] or altitude_m > levels[-1]:
        raise ValueError("source altitude is outside the radial grid")
    upper = int(np.searchsorted(levels, altitude_m, side="left"))
    if upper < len(levels) and levels[upper] == altitude_m:
        return np.asarray((upper,), dtype=np.int64), np.asarray((1.0,), dtype=np.float64)
    lower = upper - 1
    wu = (altitude_m - levels[lower]) / (levels[upper] - levels[lower])
    return np.asarray((lower, upper), dtype=np.int64), np.asarray((1.0 - wu, wu), dtype=np.float64)


@dataclass(frozen=True, slots=True)
class GaussianCurrent:
    """Vertical current with a Gaussian, optionally carrier-modulated, pulse."""

    latitude_deg: float = GWANGJU_LATITUDE_DEG
    longitude_deg: float = GWANGJU_LONGITUDE_DEG
    altitude_m: float = 2_500.0
    peak_current_a: float = 1.0e6
    vertical_element_length_m: float = 5_000.0
    center_time_s: float | None = None
    one_over_e_half_width_s: float | None = None
    carrier_frequency_hz: float = 0.0

    def __post_init__(self) -> None:
        finite = (self.latitude_deg, self.longitude_deg, self.altitude_m, self.peak_current_a, self.vertical_element_length_m, self.carrier_frequency_hz)
        if not all(np.isfinite(v) for v in finite):
            raise ValueError("source coordinates and waveform values must be finite")
        if not -90.0 <= self.latitude_deg <= 90.0:
            raise ValueError("source latitude must be in [-90, 90]")
        if self.vertical_element_length_m <= 0.0:
            raise ValueError("vertical source element length must be positive")
        if self.center_time_s is not None and not np.isfinite(self.center_time_s):
            raise ValueError("source center time must be finite")
        if self.one_over_e_half_width_s is not None and (not np.isfinite(self.one_over_e_half_width_s) or self.one_over_e_half_width_s <= 0.0):
            raise ValueError("source half width must be finite and positive")
        if self.carrier_frequency_hz < 0.0:
            raise ValueError("source carrier frequency cannot be negative")

    def direction(self) -> NDArray[np.float64]:
        return geographic_direction(self.latitude_deg, self.longitude_deg)

    def location(self, simulation) -> tuple[int, int]:
        vertex = int(np.argmax(simulation.mesh.vertices @ self.direction()))
        layer = int(np.argmin(np.abs(simulation.altitudes_m - self.altitude_m)))
        return vertex, layer

    def distribution(self, simulation):
        return geographic_distribution(simulation, self.latitude_deg, self.longitude_deg, self.altitude_m)

    def staggered_distribution(self, simulation):
        """Barycentric x radial-linear supports on Er nodes (sources.py:220-235)."""

        vertices, _, hw = self.distribution(simulation)
        layers, rw = radial_linear_distribution(simulation.altitudes_m, self.altitude_m)
        n = len(layers)
        return np.repeat(vertices, n), np.tile(layers, len(vertices)), np.repeat(hw, n) * np.tile(rw, len(vertices))

    def _envelope_parameters(self, dt_s: float) -> tuple[float, float]:
        if self.one_over_e_half_width_s is not None:
            width = self.one_over_e_half_width_s
        elif self.carrier_frequency_hz:
            width = 0.5 / self.carrier_frequency_hz
        else:
            width = 12.0 * dt_s
        centre = self.center_time_s if self.center_time_s is not None else max(4.0 * width, 36.0 * dt_s)
        return width, centre

    def current_a(self, time_s: float, dt_s: float) -> float:
        """Waveform at one instant (sources.py:237-254)."""

        width, centre = self._envelope_parameters(dt_s)
        envelope = np.exp(-(((time_s - centre) / width) ** 2))
        if self.carrier_frequency_hz:
            envelope *= np.cos(2.0 * np.pi * self.carrier_frequency_hz * (time_s - centre))
        return float(self.peak_current_a * envelope)

    def current_series(self, times_s: NDArray[np.float64], dt_s: float) -> NDArray[np.float64]:
        """The same waveform on an array of instants (one NumPy pass)."""

        width, centre = self._envelope_parameters(dt_s)
        t = np.asarray(times_s, dtype=np.float64)
        envelope = np.exp(-(((t - centre) / width) ** 2))
        if self.carrier_frequency_hz:
            envelope = envelope * np.cos(2.0 * np.pi * self.carrier_frequency_hz * (t - centre))
        return self.peak_current_a * envelope


@dataclass(frozen=True, slots=True)
class TangentialGaussianCurrent(GaussianCurrent):
    """Ground-line current projected on the containing face's edges (sources.py:257-335)."""

    altitude_m: float = 0.0
    azimuths_deg: tuple[float, ...] = (0.0,)
    line_lengths_m: tuple[float, ...] | None = None
    edge_assignment: str = "projected"

    def __post_init__(self) -> None:
        GaussianCurrent.__post_init__(self)
        if not self.azimuths_deg:
            raise ValueError("azimuths_deg must contain at least one direction")
        if not all(np.isfinite(v) for v in self.azimuths_deg):
            raise ValueError("source azimuths must be finite")
        if self.line_lengths_m is not None:
            if len(self.line_lengths_m) != len(self.azimuths_deg):
                raise ValueError("line_lengths_m must match azimuths_deg")
            if not all(np.isfinite(v) and v > 0.0 for v in self.line_lengths_m):
                raise ValueError("ground-line lengths must be finite and positive")
        if self.edge_assignment not in {"projected", "nearest"}:
            raise ValueError("edge_assignment must be 'projected' or 'nearest'")

    def edge_distribution(self, simulation):
        face = geographic_face_index(simulation, self.latitude_deg, self.longitude_deg)
        edges = simulation.mesh.face_edges[face].copy()
        ends = simulation.mesh.vertices[simulation.mesh.edges[edges]]
        dirs = ends[:, 1] - ends[:, 0]
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        east, north = geographic_tangent_basis(self.latitude_deg, self.longitude_deg)
        lengths = simulation.mesh.primal_edge_angles[edges] * (simulation.config.earth_radius_m + self.altitude_m)
        weights = np.zeros(len(edges), dtype=np.float64)
        lines = self.line_lengths_m or tuple(1.0 for _ in self.azimuths_deg)
        for az, ll in zip(self.azimuths_deg, lines, strict=True):
            a = np.deg2rad(az)
            proj = dirs @ (np.cos(a) * north + np.sin(a) * east)
            if self.edge_assignment == "projected":
                weights += ll * proj / lengths
            else:
                k = int(np.argmax(np.abs(proj)))
                weights[k] += ll * proj[k] / lengths[k]
        layers, rw = radial_linear_distribution(simulation.radial_midpoint_altitudes_m, self.altitude_m)
        return (
            np.repeat(edges, len(layers)),
            np.tile(layers, len(edges)),
            np.repeat(weights, len(layers)) * np.tile(rw, len(edges)),
        )
